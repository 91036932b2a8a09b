// ref_gpu.cu -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref{2d,3d}_gpu.so).
//
// C entry points onto the reference's own CUDA thinning library
// (2D/LibThinning2D.cu, 3D/LibThinning3D.cu), rebuilt for sm_100a from the
// reference tree and linked beside this file.  Used only as an informative
// cross-check on shapes the reference kernels handle in bounds: 2D widths up
// to 1024 (wider images read past the 2D kernel's shared-memory allocation,
// 2D/CUDA_ThinningKernelMultiBlock2D.cuh:31, or divide by zero on the host,
// 2D/LibThinning2D.cu:66), 3D dimensions that are multiples of 32 and >= 64.
#include <cstdint>
#ifdef REF_DIM3
#include "LibThinning3D.h"
extern "C" void ref3d_gpu_thin_u8(int w, int h, int d, uint8_t *in, uint8_t *out)
{
    Thinning3D<unsigned char>(w, h, d, in, out);
}
#else
#include "LibThinning2D.h"
extern "C" void ref2d_gpu_thin_u8(int w, int h, uint8_t *in, uint8_t *out)
{
    Thinning2D<unsigned char>(w, h, in, out);
}
#endif
