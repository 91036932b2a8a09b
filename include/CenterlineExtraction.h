/*
 * CenterlineExtraction.h -- drop-in for the reference's 2D centreline entry
 * point (2D/CenterlineExtraction.h:25-28).  Same signature and ownership:
 * *out_x, *out_y and *out_idx are allocated with new[] and the caller
 * delete[]s them.  out_idx has nsegs+1 entries (out_idx[nsegs] = number of
 * points); the return value is the number of segments.
 *
 * Thinning and segment extraction run on the GPU; pruning removes end
 * segments with at most max_segment_length points; smoothing is a moving
 * average of half-width smoothing_span.  The image should have no
 * foreground on its outer 1-pixel frame (as for the reference).  On failure
 * the function returns 0 with empty (but valid, delete[]-able) outputs and
 * bgt_last_error() describes the failure.
 */
#pragma once

template <typename PixelType>
unsigned int CenterlineExtraction(PixelType *data, int width, int height, int max_segment_length,
                                  int smoothing_span, float **out_x, float **out_y, unsigned int **out_idx);
