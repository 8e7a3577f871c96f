// lpc.cuh - host launchers of the learned-preconditioner and flexible-CG kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cfd2d_b200.h"

namespace cfd {
namespace lpc {

size_t conv32_smem_bytes(int rows);
cudaError_t conv32_tc(const __nv_bfloat16* x, const __nv_bfloat16* wpack, const float* bias,
                      const __nv_bfloat16* skip, const uint8_t* mask, __nv_bfloat16* y, int H, int W, int relu,
                      int* err, cudaStream_t s);
cudaError_t pack_w32(const float* w, __nv_bfloat16* img, int adjoint, cudaStream_t s);
cudaError_t conv_generic(int cin, int cout, const void* x, int xbf, const float* w, const float* bias,
                         const uint8_t* mask, void* y, int ybf, int H, int W, int relu, int transposed,
                         cudaStream_t s);
cudaError_t pool2(const __nv_bfloat16* x, __nv_bfloat16* y, int H, int W, cudaStream_t s);
cudaError_t pool_mask(const uint8_t* m, uint8_t* mc, int H, int W, cudaStream_t s);
cudaError_t upadd(const __nv_bfloat16* coarse, const __nv_bfloat16* skip, __nv_bfloat16* y, int H, int W, float scale,
                  cudaStream_t s);
cudaError_t relu_bwd(const float* dy, const __nv_bfloat16* y, const uint8_t* mask, float* g, int npix, int ch,
                     int relu, cudaStream_t s);
cudaError_t upadd_bwd(const float* dy, float* dcoarse, int H, int W, float scale, cudaStream_t s);
cudaError_t pool_bwd(const float* dcoarse, float* dfine, int H, int W, cudaStream_t s);
size_t conv_dw_partial_floats(int cin, int cout, int H, int W, int pix_per_block);
cudaError_t conv_dw(int cin, int cout, const void* x, int xbf, const float* g, int H, int W, int pix_per_block,
                    float* partial, float* out, cudaStream_t s);

}  // namespace lpc

namespace fcg {

using FcgScalars = cfd2d_fcg_scalars;

size_t partial_doubles(int n);
cudaError_t init(const cfd2d_poisson& op, const double* F, const double* G, const double* rhs, double dx,
                 double dy, const double* dt_ptr, double* b, double* x, double* r, double* p_zero, FcgScalars* s,
                 double* partial, cudaStream_t st);
cudaError_t pq(const cfd2d_poisson& op, const double* p, double* q, const double* r, FcgScalars* s,
               double* partial, cudaStream_t st);
cudaError_t update(int n, double* x, double* r, const double* p, const double* q, FcgScalars* s, double* partial,
                   cudaStream_t st);
cudaError_t zr(int n, const double* z, const double* q, int first, FcgScalars* s, double* partial,
               cudaStream_t st);
cudaError_t dir(int n, const double* z, double* p, const FcgScalars* s, cudaStream_t st);
cudaError_t net_in(int n, const double* r, const FcgScalars* s, const uint8_t* mask, float* in, cudaStream_t st);
cudaError_t net_out(int n, const float* out, const double* r, const double* dinv, const uint8_t* mask,
                    const FcgScalars* s, double scale, double jacobi, double* z, cudaStream_t st);
cudaError_t scatter_p(const cfd2d_poisson& op, const double* x, double* p_pad, cudaStream_t st);
cudaError_t gate(const FcgScalars* s, cfd2d_fcg_control* ctl, unsigned long long handle, cudaStream_t st);
cudaError_t zero_rhs(int n, const double* b, double* x, const FcgScalars* s, cudaStream_t st);

}  // namespace fcg
}  // namespace cfd
