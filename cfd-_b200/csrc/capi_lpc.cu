// capi_lpc.cu - extern "C" entry points of the learned preconditioner and the
// flexible CG (declared in include/cfd2d_b200.h; no counterpart in the reference).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/cfd2d_b200.h"
#include "lpc.cuh"

using namespace cfd;

namespace {
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int status_of(cudaError_t e) { return e == cudaSuccess ? CFD2D_OK : CFD2D_E_CUDA; }
inline const __nv_bfloat16* bf(const void* p) { return reinterpret_cast<const __nv_bfloat16*>(p); }
inline __nv_bfloat16* bfw(void* p) { return reinterpret_cast<__nv_bfloat16*>(p); }
bool hw_ok(int H, int W) { return H >= 1 && W >= 1 && (long long)H * W < (1LL << 30); }
}  // namespace

extern "C" {

size_t cfd2d_lpc_w32_bytes(void) { return (size_t)32 * 288 * 2; }

int cfd2d_lpc_pack_w32(const float* w, void* image, void* stream) {
    if (!w || !image) return CFD2D_E_ARG;
    return status_of(lpc::pack_w32(w, bfw(image), 0, as_stream(stream)));
}

int cfd2d_lpc_pack_w32_adjoint(const float* w, void* image, void* stream) {
    if (!w || !image) return CFD2D_E_ARG;
    return status_of(lpc::pack_w32(w, bfw(image), 1, as_stream(stream)));
}

int cfd2d_lpc_conv32(const void* x, const void* image, const float* bias, const void* skip,
                     const uint8_t* mask, void* y, int H, int W, int relu, int32_t* err, void* stream) {
    if (!x || !image || !bias || !y || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::conv32_tc(bf(x), bf(image), bias, bf(skip), mask, bfw(y), H, W, relu,
                                    reinterpret_cast<int*>(err), as_stream(stream)));
}

int cfd2d_lpc_conv(int cin, int cout, const void* x, int x_bf16, const float* w, const float* bias,
                   const uint8_t* mask, void* y, int y_bf16, int H, int W, int relu, int transposed,
                   void* stream) {
    if (!x || !w || !y || !hw_ok(H, W)) return CFD2D_E_ARG;
    if (!((cin == 1 || cin == 32) && (cout == 1 || cout == 32)) || (cin == 1 && cout == 1)) return CFD2D_E_ARG;
    return status_of(lpc::conv_generic(cin, cout, x, x_bf16, w, bias, mask, y, y_bf16, H, W, relu, transposed,
                                       as_stream(stream)));
}

int cfd2d_lpc_pool2(const void* x, void* y, int H, int W, void* stream) {
    if (!x || !y || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::pool2(bf(x), bfw(y), H, W, as_stream(stream)));
}

int cfd2d_lpc_pool_mask(const uint8_t* m, uint8_t* mc, int H, int W, void* stream) {
    if (!m || !mc || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::pool_mask(m, mc, H, W, as_stream(stream)));
}

int cfd2d_lpc_upadd(const void* coarse, const void* skip, void* y, int H, int W, float scale, void* stream) {
    if (!coarse || !skip || !y || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::upadd(bf(coarse), bf(skip), bfw(y), H, W, scale, as_stream(stream)));
}

int cfd2d_lpc_relu_bwd(const float* dy, const void* y, const uint8_t* mask, float* g, int npix, int ch,
                       int relu, void* stream) {
    if (!dy || !g || (relu && !y) || npix < 1) return CFD2D_E_ARG;
    return status_of(lpc::relu_bwd(dy, bf(y), mask, g, npix, ch, relu, as_stream(stream)));
}

int cfd2d_lpc_upadd_bwd(const float* dy, float* dcoarse, int H, int W, float scale, void* stream) {
    if (!dy || !dcoarse || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::upadd_bwd(dy, dcoarse, H, W, scale, as_stream(stream)));
}

int cfd2d_lpc_pool_bwd(const float* dcoarse, float* dfine, int H, int W, void* stream) {
    if (!dcoarse || !dfine || !hw_ok(H, W)) return CFD2D_E_ARG;
    return status_of(lpc::pool_bwd(dcoarse, dfine, H, W, as_stream(stream)));
}

size_t cfd2d_lpc_conv_dw_partial_floats(int cin, int cout, int H, int W, int pix_per_block) {
    return lpc::conv_dw_partial_floats(cin, cout, H, W, pix_per_block);
}

int cfd2d_lpc_conv_dw(int cin, int cout, const void* x, int x_bf16, const float* g, int H, int W,
                      int pix_per_block, float* partial, float* out, void* stream) {
    if (!x || !g || !partial || !out || !hw_ok(H, W) || pix_per_block < 1) return CFD2D_E_ARG;
    return status_of(lpc::conv_dw(cin, cout, x, x_bf16, g, H, W, pix_per_block, partial, out, as_stream(stream)));
}

size_t cfd2d_fcg_partial_doubles(int n) { return fcg::partial_doubles(n); }

int cfd2d_fcg_init(const cfd2d_poisson* op, const double* F, const double* G, const double* rhs, double dx,
                   double dy, const double* dt, double* b, double* x, double* r, double* p_zero,
                   cfd2d_fcg_scalars* s, double* partial, void* stream) {
    if (!op || !b || !x || !r || !s || !partial || (!rhs && (!F || !G))) return CFD2D_E_ARG;
    return status_of(fcg::init(*op, F, G, rhs, dx, dy, dt, b, x, r, p_zero, s, partial, as_stream(stream)));
}

int cfd2d_fcg_pq(const cfd2d_poisson* op, const double* p, double* q, const double* r, cfd2d_fcg_scalars* s,
                 double* partial, void* stream) {
    if (!op || !p || !q || !r || !s || !partial) return CFD2D_E_ARG;
    return status_of(fcg::pq(*op, p, q, r, s, partial, as_stream(stream)));
}

int cfd2d_fcg_update(int n, double* x, double* r, const double* p, const double* q, cfd2d_fcg_scalars* s,
                     double* partial, void* stream) {
    if (n < 1 || !x || !r || !p || !q || !s || !partial) return CFD2D_E_ARG;
    return status_of(fcg::update(n, x, r, p, q, s, partial, as_stream(stream)));
}

int cfd2d_fcg_zr(int n, const double* z, const double* q, int first, cfd2d_fcg_scalars* s, double* partial,
                 void* stream) {
    if (n < 1 || !z || !q || !s || !partial) return CFD2D_E_ARG;
    return status_of(fcg::zr(n, z, q, first, s, partial, as_stream(stream)));
}

int cfd2d_fcg_dir(int n, const double* z, double* p, const cfd2d_fcg_scalars* s, void* stream) {
    if (n < 1 || !z || !p || !s) return CFD2D_E_ARG;
    return status_of(fcg::dir(n, z, p, s, as_stream(stream)));
}

int cfd2d_fcg_net_in(int n, const double* r, const cfd2d_fcg_scalars* s, const uint8_t* mask, float* in,
                     void* stream) {
    if (n < 1 || !r || !s || !mask || !in) return CFD2D_E_ARG;
    return status_of(fcg::net_in(n, r, s, mask, in, as_stream(stream)));
}

int cfd2d_fcg_net_out(int n, const float* out, const double* r, const double* dinv, const uint8_t* mask,
                      const cfd2d_fcg_scalars* s, double scale, double jacobi, double* z, void* stream) {
    if (n < 1 || !out || !r || !dinv || !mask || !s || !z) return CFD2D_E_ARG;
    return status_of(fcg::net_out(n, out, r, dinv, mask, s, scale, jacobi, z, as_stream(stream)));
}

int cfd2d_fcg_scatter_p(const cfd2d_poisson* op, const double* x, double* p_padded, void* stream) {
    if (!op || !x || !p_padded) return CFD2D_E_ARG;
    return status_of(fcg::scatter_p(*op, x, p_padded, as_stream(stream)));
}

int cfd2d_fcg_gate(const cfd2d_fcg_scalars* s, cfd2d_fcg_control* ctl, uint64_t handle, void* stream) {
    if (!s || !ctl) return CFD2D_E_ARG;
    return status_of(fcg::gate(s, ctl, (unsigned long long)handle, as_stream(stream)));
}

int cfd2d_fcg_zero_rhs(int n, const double* b, double* x, const cfd2d_fcg_scalars* s, void* stream) {
    if (n < 1 || !b || !x || !s) return CFD2D_E_ARG;
    return status_of(fcg::zero_rhs(n, b, x, s, as_stream(stream)));
}

int cfd2d_capture_begin(void* stream) {
    if (!stream) return CFD2D_E_ARG;  // the legacy default stream cannot be captured
    return status_of(cudaStreamBeginCapture(as_stream(stream), cudaStreamCaptureModeRelaxed));
}

int cfd2d_capture_condition(void* stream, uint64_t* handle_out) {
    if (!stream || !handle_out) return CFD2D_E_ARG;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(as_stream(stream), &cs, nullptr, &g, nullptr, nullptr);
    if (e != cudaSuccess) return status_of(e);
    if (cs != cudaStreamCaptureStatusActive || !g) return CFD2D_E_ARG;
    cudaGraphConditionalHandle h = 0;
    e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return status_of(e);
    *handle_out = (uint64_t)h;
    return CFD2D_OK;
}

int cfd2d_capture_while_begin(void* stream, void* body_stream, uint64_t handle) {
    if (!stream || !body_stream || !handle || stream == body_stream) return CFD2D_E_ARG;
    cudaStream_t s = as_stream(stream);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps);
    if (e != cudaSuccess) return status_of(e);
    if (cs != cudaStreamCaptureStatusActive || !g) return CFD2D_E_ARG;
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = (cudaGraphConditionalHandle)handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, g, deps, ndeps, &np);
    if (e != cudaSuccess) return status_of(e);
    e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return status_of(e);
    cudaGraph_t body = np.conditional.phGraph_out[0];
    return status_of(cudaStreamBeginCaptureToGraph(as_stream(body_stream), body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed));
}

int cfd2d_capture_while_end(void* body_stream) {
    if (!body_stream) return CFD2D_E_ARG;
    cudaGraph_t body = nullptr;
    return status_of(cudaStreamEndCapture(as_stream(body_stream), &body));
}

int cfd2d_capture_end(void* stream, void** graph_out) {
    if (!stream || !graph_out) return CFD2D_E_ARG;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(as_stream(stream), &g);
    if (e != cudaSuccess) return status_of(e);
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return status_of(e);
    *graph_out = (void*)x;
    return CFD2D_OK;
}

int cfd2d_capture_abort(void* stream) {
    if (!stream) return CFD2D_E_ARG;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(as_stream(stream), &cs) != cudaSuccess) {
        cudaGetLastError();
        return CFD2D_E_CUDA;
    }
    if (cs == cudaStreamCaptureStatusNone) return CFD2D_OK;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(as_stream(stream), &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return CFD2D_OK;
}

}  // extern "C"
