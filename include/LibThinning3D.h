/*
 * LibThinning3D.h -- drop-in for the reference's 3D thinning entry point
 * (3D/LibThinning3D.h:14-15).  Same signature; link with libbgt.so.
 *
 * data and out are host arrays of width*height*depth voxels,
 * data[(z*height + y)*width + x].  The reference requires every dimension to
 * be a multiple of 32 and at least 64 (3D/LibThinning3D.h:13,
 * 3D/LibThinning3D.cu:50); this implementation accepts any size >= 1 and
 * writes every output voxel (the reference copies only width*height*depth
 * bytes back whatever the pixel type, 3D/LibThinning3D.cu:81).  Explicit
 * instantiations: unsigned char, unsigned short, unsigned int, char, short,
 * int, float, bool.
 */
#pragma once

template <typename PixelType>
void Thinning3D(int width, int height, int depth, PixelType *data, PixelType *out);
