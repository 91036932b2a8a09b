/*
 * LibThinning2D.h -- drop-in for the reference's 2D thinning entry point
 * (2D/LibThinning2D.h:14-15).  Same signature; link with libbgt.so.
 *
 * data and out are host arrays of width*height pixels, row-major.  Unlike
 * the reference, any width/height >= 1 is accepted (the reference pads to a
 * power-of-two width internally and divides by zero at width 4096,
 * 2D/LibThinning2D.cu:66).  Output pixels are 0/1.  Explicit instantiations:
 * unsigned char, unsigned short, unsigned int, char, signed char, short, int,
 * float, double, bool.  On a CUDA error the output is zero-filled and
 * bgt_last_error() (bgt_capi.h) describes the failure.
 */
#pragma once

template <typename PixelType>
void Thinning2D(int width, int height, PixelType *data, PixelType *out);
