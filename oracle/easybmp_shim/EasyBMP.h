/*
 * No-op stand-in for the EasyBMP header, used only to compile the reference
 * fdtd3d CPU build (the oracle binary under oracle/_ref).  The reference's
 * CMake downloads EasyBMP at configure time; there is no network here, and
 * the FDTD arithmetic never depends on it.  Every image call is accepted and
 * does nothing, so BMP output is simply not produced.  Field parity uses the
 * reference's TXT dumper instead.
 *
 * Declares only the members the reference's File-Management sources call:
 * RGBApixel {Blue, Green, Red, Alpha}, BMP::SetSize, SetBitDepth,
 * WriteToFile, ReadFromFile, SetPixel, GetPixel, TellWidth, TellHeight.
 */
#ifndef ORACLE_EASYBMP_SHIM_H
#define ORACLE_EASYBMP_SHIM_H

/* The real header pulls these in, and the reference's loaders rely on it. */
#include <iostream>
#include <cmath>
#include <cctype>
#include <cstring>
#include <cstdio>

typedef unsigned char ebmpBYTE;

struct RGBApixel
{
  ebmpBYTE Blue;
  ebmpBYTE Green;
  ebmpBYTE Red;
  ebmpBYTE Alpha;
  RGBApixel () : Blue (0), Green (0), Red (0), Alpha (0) {}
};

class BMP
{
  int width;
  int height;
public:
  BMP () : width (1), height (1) {}
  bool SetSize (int w, int h) { width = w; height = h; return true; }
  bool SetBitDepth (int) { return true; }
  bool WriteToFile (const char *) { return true; }
  bool ReadFromFile (const char *) { return true; }
  bool SetPixel (int, int, RGBApixel) { return true; }
  RGBApixel GetPixel (int, int) const { return RGBApixel (); }
  int TellWidth () const { return width; }
  int TellHeight () const { return height; }
};

#endif /* ORACLE_EASYBMP_SHIM_H */
