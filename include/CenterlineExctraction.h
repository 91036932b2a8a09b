/*
 * CenterlineExctraction.h -- drop-in for the reference's 3D centreline entry
 * point (3D/CenterlineExctraction.h:26-29; the file name keeps the
 * reference's spelling so existing #include lines work; CenterlineExtraction3D.h
 * includes this file).  Same signature and ownership as the reference:
 * outputs allocated with new[], caller delete[]s them; returns the number of
 * segments.  Volumes of any size are padded internally to multiples of 32
 * with background (the reference leaves that padding uninitialised,
 * 3D/CenterlineExtraction.cpp:32).
 */
#pragma once

template <typename PixelType>
unsigned int CenterlineExtraction(PixelType *data, int width, int height, int depth, int max_segment_length,
                                  int smoothing_span, float **out_x, float **out_y, float **out_z,
                                  unsigned int **out_idx);
