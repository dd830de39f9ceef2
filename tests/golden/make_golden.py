"""Regenerates the golden fixtures in this directory (run in a container that
has the reference sources; not needed at test time).

* exhy_1d_unit_test.json - the 1-D ExHy Ex values that the reference's own
  unit test hard-codes after 200 TF/SF steps (E_CENTERED, SIZE 20, TFSF 7,
  DX 0.002, LAMBDA 0.2), extracted as text from
  Source/UnitTests/unit-test-internalscheme.cpp (test1D_ExHy, E_CENTERED
  block).
* unit_test_1d_modes.json - the same unit test's golden blocks for all six
  1-D modes (test1D_ExHy .. test1D_EzHy), E_CENTERED and H_CENTERED, real
  (sine source) and imaginary (cosine source) parts.
* ref_*.npz - fields dumped by the reference CPU double build
  (oracle/_ref/fdtd3d, built from the reference sources by oracle/Makefile)
  on small seeded configurations, with the run arguments stored alongside.

    python tests/golden/make_golden.py [/path/to/fdtd3d/source/tree]
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import run_reference  # noqa: E402

CASES = {
    "ref_dim3_ps": dict(mode=3, size=12, point_source=(6, 6, 6), point_source_mask=1 << 2,
                        teta=0, phi=0, psi=0, steps=15),
    "ref_dim3_pml_tfsf": dict(mode=3, size=14, use_pml=True, pml=3, use_tfsf=True, tfsf_left=5, tfsf_right=5,
                              teta=30, phi=45, psi=0, steps=25),
    "ref_dim3_drude": dict(mode=3, size=12, use_pml=True, pml=2, use_tfsf=True, tfsf_left=4, tfsf_right=4,
                           teta=0, phi=0, psi=0, use_metamaterials=True, steps=20),
    "ref_tmz_pml_tfsf": dict(mode=2, size=(32, 32), use_pml=True, pml=6, use_tfsf=True, tfsf_left=10,
                             tfsf_right=10, teta=90, phi=30, psi=90, steps=50),
    # H_CENTERED (--layout-type 1)
    "ref_dim3_hc_pml_tfsf": dict(mode=3, size=14, use_pml=True, pml=3, use_tfsf=True, tfsf_left=5, tfsf_right=5,
                                 teta=30, phi=45, psi=10, steps=25, layout=1),
    "ref_tez_hc_pml_tfsf": dict(mode=6, size=(30, 28), use_pml=True, pml=5, use_tfsf=True, tfsf_left=9,
                                tfsf_right=8, teta=90, phi=35, psi=0, steps=40, layout=1),
}


def materials_for(name):
    if name in ("ref_dim3_pml_tfsf", "ref_dim3_hc_pml_tfsf"):
        x, y, z = np.indices((14, 14, 14))
        return {"eps": np.where((x - 7) ** 2 + (y - 7) ** 2 + (z - 7) ** 2 < 9, 4.0, 1.0)}
    if name == "ref_dim3_drude":
        om = np.zeros((12, 12, 12))
        ga = np.zeros((12, 12, 12))
        om[:, :, 5:8] = np.float32(2 * np.pi * 30e9)
        ga[:, :, 5:8] = np.float32(2 * np.pi * 1e9)
        return {"omegape": om, "gammae": ga, "omegapm": om, "gammam": ga}
    if name == "ref_tez_hc_pml_tfsf":
        x, y = np.indices((30, 28))
        return {"eps": np.where((x - 15) ** 2 + (y - 14) ** 2 < 30, 3.0, 1.0)}
    return None


def extract_exhy(src_root):
    path = os.path.join(src_root, "Source", "UnitTests", "unit-test-internalscheme.cpp")
    text = open(path).read()
    block = text.split("if (SOLVER_SETTINGS.getDoUseTFSF () && layout_type == E_CENTERED)")[1]
    block = block.split("if (SOLVER_SETTINGS.getDoUseTFSF () && layout_type == H_CENTERED)")[0]
    vals = {}
    for m in re.finditer(r"FIELDVALUE \(([-0-9.e]+), ([-0-9.e]+)\), GRID_COORDINATE_1D \((\d+), ct1\)", block):
        vals[int(m.group(3))] = [float(m.group(1)), float(m.group(2))]
    return {"size": 20, "tfsf": 7, "dx": 0.002, "wavelength": 0.2, "courant": 0.5, "steps": 200,
            "source": "Source/UnitTests/unit-test-internalscheme.cpp (test1D_ExHy, E_CENTERED)",
            "ex": {str(k): v for k, v in sorted(vals.items())}}


def extract_1d_modes(src_root):
    """Every 1-D mode's golden block of the same unit test, both layouts: the
    run axis, the three angles, the compared E component and its
    (sine, cosine) values after 200 TF/SF steps.  The complex build of the
    test compares the real part with a sine source and the imaginary part
    with a cosine source."""
    path = os.path.join(src_root, "Source", "UnitTests", "unit-test-internalscheme.cpp")
    text = open(path).read()
    out = {}
    for m in re.finditer(r"void test1D_(\w\w\w\w) \(\)\n\{(.*?)\n\}\n", text, re.S):
        name, body = m.group(1), m.group(2)
        axis = re.search(r"CoordinateType ct1 = CoordinateType::([XYZ]);", body).group(1)
        angles = [float(re.search(r"FPValue angle%d = ([-0-9.]+);" % i, body).group(1)) for i in (1, 2, 3)]
        comp = re.search(r"test1D \(intScheme\.get(\w\w) \(\)", body).group(1)
        entry = {"axis": "XYZ".index(axis), "teta": angles[0], "phi": angles[1], "psi": angles[2],
                 "component": comp}
        for layout in ("E_CENTERED", "H_CENTERED"):
            block = body.split("if (SOLVER_SETTINGS.getDoUseTFSF () && layout_type == %s)" % layout)[1]
            block = block.split("}")[0]
            vals = {}
            for v in re.finditer(r"FIELDVALUE \(([-0-9.e]+), ([-0-9.e]+)\), GRID_COORDINATE_1D \((\d+), ct1\)",
                                 block):
                vals[str(int(v.group(3)))] = [float(v.group(1)), float(v.group(2))]
            assert len(vals) == 20, (name, layout, len(vals))
            entry[layout] = vals
        out[name] = entry
    assert len(out) == 6, sorted(out)
    return {"size": 20, "tfsf": 7, "dx": 0.002, "wavelength": 0.2, "courant": 0.5, "steps": 200,
            "source": "Source/UnitTests/unit-test-internalscheme.cpp (test1D_*, both layouts)", "modes": out}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference source root>")
    src_root = sys.argv[1]
    with open(os.path.join(HERE, "exhy_1d_unit_test.json"), "w") as f:
        json.dump(extract_exhy(src_root), f, indent=1)
    with open(os.path.join(HERE, "unit_test_1d_modes.json"), "w") as f:
        json.dump(extract_1d_modes(src_root), f, indent=1)
    for name, kw in CASES.items():
        mats = materials_for(name)
        fields, _ = run_reference(materials=mats, **kw)
        extra = {f"mat_{k}": v for k, v in (mats or {}).items()}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), args=json.dumps(kw),
                            **{k: v for k, v in fields.items()}, **extra)
        print(name, {k: float(np.abs(v).max()) for k, v in fields.items()})


if __name__ == "__main__":
    main()
