// fcg.cu - flexible conjugate gradients around a variable preconditioner, for the
// learned Poisson preconditioner. The form is Notay's FCG with one stored
// direction: beta = -(z . A p_old) / (p_old . A p_old), alpha = (p . r) / (p . A p).
// Unlike the Polak-Ribiere form it relies on no positivity of r . M(r): every step
// is an exact line search along p, so the A-norm of the error never grows. Vectors are FP64 over the
// nx*ny interior cells; the operator is the matrix-free 5-point A of the
// pressure solver (same data as cfd2d_poisson, same row summation order). Every
// scalar (alpha, beta, r.z, ||r||^2) stays on the device: each reduction kernel
// writes per-block partials and its last block adds them in block order.
#include <cuda_runtime.h>
#include <math.h>

#include "device.cuh"
#include "lpc.cuh"

namespace cfd {
namespace fcg {

namespace {
constexpr int T = 256;

__device__ __forceinline__ double row_sum(bool periodic, int i, int nx, double tW, double tS, double tC,
                                          double tN, double tE) {
    if (periodic && i == 0) return (((tS + tC) + tN) + tE) + tW;
    if (periodic && i == nx - 1) return (((tE + tW) + tS) + tC) + tN;
    return (((tW + tS) + tC) + tN) + tE;
}

__device__ __forceinline__ double apply_A(const cfd2d_poisson& op, const double* X, int c) {
    const int nx = op.nx, ny = op.ny;
    const int i = c / ny, j = c % ny;
    const uint8_t nb = op.nbr[c];
    if (!(nb & 0x80)) return 0.0;
    double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
    if (nb & 2) tS = -op.dy2 * X[c - 1];
    if (nb & 4) tN = -op.dy2 * X[c + 1];
    if (nb & 1) tW = -op.dx2 * X[((i == 0) ? nx - 1 : i - 1) * ny + j];
    if (nb & 8) tE = -op.dx2 * X[((i == nx - 1) ? 0 : i + 1) * ny + j];
    return row_sum(op.periodic != 0, i, nx, tW, tS, op.diag[c] * X[c], tN, tE);
}

// K block sums -> partial[k * gridDim.x + block]; the last block adds them in block
// order into tot[0..K); returns true in the last block (thread 0 holds the totals)
template <int K>
__device__ __forceinline__ bool reduce_last(double (&v)[K], double* partial, unsigned int* ticket,
                                            double (&tot)[K]) {
    __shared__ double sred[32 * K];
    block_sum<K>(v, sred);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) partial[k * gridDim.x + blockIdx.x] = v[k];
    if (!last_block(ticket)) return false;
    double t[K];
    for (int k = 0; k < K; ++k) {
        t[k] = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t[k] += __ldcg(&partial[k * gridDim.x + b]);
    }
    block_sum<K>(t, sred);
    for (int k = 0; k < K; ++k) tot[k] = t[k];
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

}  // namespace

// b = -(div(F, G) / dt) on fluid cells (no Neumann component: the learned path runs
// on domains with an outflow boundary), r = b - A x, ||b||^2, ||r||^2
__global__ void k_init(cfd2d_poisson op, const double* F, const double* G, const double* rhs, double dx,
                       double dy, const double* dt_ptr, double* b, double* x, double* r, double* p_zero,
                       FcgScalars* s, double* partial) {
    const int n = op.nx * op.ny;
    const int ny = op.ny;
    double v[2] = {0.0, 0.0};
    const double dt = dt_ptr ? *dt_ptr : 1.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double bb = 0.0;
        if (op.nbr[c] & 0x80) {
            if (rhs) {
                bb = -rhs[c];
            } else {
                const int i = c / ny, j = c % ny;
                const int pu = ny + 2, pv = ny + 1, ig = i + 1, jg = j + 1;
                const double div = (F[ig * pu + jg] - F[(ig - 1) * pu + jg]) / dx +
                                   (G[ig * pv + jg] - G[ig * pv + jg - 1]) / dy;
                bb = -(div / dt);
            }
        }
        b[c] = bb;
        if (p_zero) p_zero[c] = 0.0;  // the first direction is z + 0 * p
        v[0] += bb * bb;
    }
    double tot[2];
    (void)tot;
    // r needs x of neighbours only (read-only here)
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double rr = (op.nbr[c] & 0x80) ? b[c] - apply_A(op, x, c) : 0.0;
        r[c] = rr;
        v[1] += rr * rr;
    }
    if (reduce_last<2>(v, partial, &s->ticket, tot) && threadIdx.x == 0) {
        s->bb = tot[0];
        s->rr = tot[1];
        s->iters = 0;
    }
}

// q = A p, alpha = (p . r) / (p . q)
__global__ void k_pq(cfd2d_poisson op, const double* p, double* q, const double* r, FcgScalars* s,
                     double* partial) {
    const int n = op.nx * op.ny;
    double v[2] = {0.0, 0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double qq = apply_A(op, p, c);
        q[c] = qq;
        v[0] += p[c] * qq;
        v[1] += p[c] * r[c];
    }
    double tot[2];
    if (reduce_last<2>(v, partial, &s->ticket, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        s->rz = tot[1];
        s->alpha = tot[1] / tot[0];
    }
}

// x += alpha p, r -= alpha q, ||r||^2
__global__ void k_update(int n, double* x, double* r, const double* p, const double* q, FcgScalars* s,
                         double* partial) {
    const double alpha = s->alpha;
    double v[1] = {0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        x[c] = x[c] + alpha * p[c];
        const double rn = r[c] - alpha * q[c];
        r[c] = rn;
        v[0] += rn * rn;
    }
    double tot[1];
    if (reduce_last<1>(v, partial, &s->ticket, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->iters = s->iters + 1;
    }
}

// beta = -(z . q_old) / (p_old . q_old) with q_old = A p_old (0 on the first direction)
__global__ void k_zr(int n, const double* z, const double* q, int first_flag, FcgScalars* s, double* partial) {
    // first_flag < 0: the first direction is the one taken before any update (iters == 0)
    const int first = first_flag < 0 ? (s->iters == 0) : first_flag;
    double v[1] = {0.0};
    if (!first)
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) v[0] += z[c] * q[c];
    double tot[1];
    if (reduce_last<1>(v, partial, &s->ticket, tot) && threadIdx.x == 0) s->beta = first ? 0.0 : -tot[0] / s->pq;
}

// p = z + beta p
__global__ void k_dir(int n, const double* z, double* p, const FcgScalars* s) {
    const double beta = s->beta;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        p[c] = z[c] + beta * p[c];
}

// preconditioner input: r / ||r|| as FP32 (masked); output: z = out * ||r|| (FP64)
__global__ void k_net_in(int n, const double* r, const FcgScalars* s, const uint8_t* mask, float* in) {
    const double inv = 1.0 / sqrt(s->rr > 0.0 ? s->rr : 1.0);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        in[c] = mask[c] ? (float)(r[c] * inv) : 0.0f;
}

// z = ||r|| * scale * out + jacobi * r / diag, masked. The network works on the
// dimensionless operator h^2 A, so scale = h^2 maps its output back to A^-1 r; the
// Jacobi term keeps the high frequencies the network does not resolve.
__global__ void k_net_out(int n, const float* out, const double* r, const double* dinv, const uint8_t* mask,
                          const FcgScalars* s, double scale, double jacobi, double* z) {
    const double sc = sqrt(s->rr > 0.0 ? s->rr : 1.0) * scale;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        z[c] = mask[c] ? ((double)out[c] * sc + jacobi * dinv[c] * r[c]) : 0.0;
}

// Stop tests of the device-driven loop, one thread: records ||r|| of this iterate,
// decides whether another iteration runs and sets the loop's graph condition.
__global__ void k_gate(const FcgScalars* s, cfd2d_fcg_control* ctl, cudaGraphConditionalHandle h) {
    const int it = s->iters;
    const int calls = ctl->calls + 1;
    ctl->calls = calls;
    const double res = sqrt(s->rr);
    if (it >= 0 && it <= ctl->maxiter) ctl->hist[it] = res;
    const double atol = ctl->rtol * sqrt(s->bb);
    int reason = CFD2D_FCG_RUNNING;
    if (!isfinite(res)) {
        reason = CFD2D_FCG_NONFINITE;
    } else if (res < atol || s->bb == 0.0) {
        reason = CFD2D_FCG_CONVERGED;
    } else if (it >= ctl->maxiter || calls > ctl->maxiter + 1) {
        reason = CFD2D_FCG_MAXITER;
    } else if (it >= ctl->stall_window && res > ctl->stall_factor * ctl->hist[it - ctl->stall_window]) {
        reason = CFD2D_FCG_STALLED;
    }
    ctl->reason = reason;
    ctl->iters = it;
    if (ctl->iters_out) *ctl->iters_out = it;
    if (h) cudaGraphSetConditional(h, reason == CFD2D_FCG_RUNNING ? 1u : 0u);
}

// x = b where ||b|| = 0 (scipy returns b for a zero right-hand side)
__global__ void k_zero_rhs(int n, const double* b, double* x, const FcgScalars* s) {
    if (s->bb != 0.0) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) x[c] = b[c];
}

// padded pressure output p[(i+1)(ny+2) + j+1] = x (no Neumann component to remove)
__global__ void k_scatter_p(cfd2d_poisson op, const double* x, double* p_pad) {
    const int nx = op.nx, ny = op.ny, pp = ny + 2;
    const int n = (nx + 2) * pp;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int i = e / pp, j = e % pp;
        double v = 0.0;
        if (i >= 1 && i <= nx && j >= 1 && j <= ny) {
            const int c = (i - 1) * ny + (j - 1);
            v = (op.nbr[c] & 0x80) ? x[c] : 0.0;
        }
        p_pad[e] = v;
    }
}

namespace {
int blocks(int n) {
    int b = (n + T - 1) / T;
    return b > 2 * 148 ? 2 * 148 : (b < 1 ? 1 : b);
}
}  // namespace

size_t partial_doubles(int n) { return (size_t)2 * blocks(n) + 8; }

cudaError_t init(const cfd2d_poisson& op, const double* F, const double* G, const double* rhs, double dx,
                 double dy, const double* dt_ptr, double* b, double* x, double* r, double* p_zero, FcgScalars* s,
                 double* partial, cudaStream_t st) {
    const int n = op.nx * op.ny;
    k_init<<<blocks(n), T, 0, st>>>(op, F, G, rhs, dx, dy, dt_ptr, b, x, r, p_zero, s, partial);
    return cudaGetLastError();
}

cudaError_t pq(const cfd2d_poisson& op, const double* p, double* q, const double* r, FcgScalars* s,
               double* partial, cudaStream_t st) {
    const int n = op.nx * op.ny;
    k_pq<<<blocks(n), T, 0, st>>>(op, p, q, r, s, partial);
    return cudaGetLastError();
}

cudaError_t update(int n, double* x, double* r, const double* p, const double* q, FcgScalars* s, double* partial,
                   cudaStream_t st) {
    k_update<<<blocks(n), T, 0, st>>>(n, x, r, p, q, s, partial);
    return cudaGetLastError();
}

cudaError_t zr(int n, const double* z, const double* q, int first, FcgScalars* s, double* partial,
               cudaStream_t st) {
    k_zr<<<blocks(n), T, 0, st>>>(n, z, q, first, s, partial);
    return cudaGetLastError();
}

cudaError_t dir(int n, const double* z, double* p, const FcgScalars* s, cudaStream_t st) {
    k_dir<<<blocks(n), T, 0, st>>>(n, z, p, s);
    return cudaGetLastError();
}

cudaError_t net_in(int n, const double* r, const FcgScalars* s, const uint8_t* mask, float* in, cudaStream_t st) {
    k_net_in<<<blocks(n), T, 0, st>>>(n, r, s, mask, in);
    return cudaGetLastError();
}

cudaError_t net_out(int n, const float* out, const double* r, const double* dinv, const uint8_t* mask,
                    const FcgScalars* s, double scale, double jacobi, double* z, cudaStream_t st) {
    k_net_out<<<blocks(n), T, 0, st>>>(n, out, r, dinv, mask, s, scale, jacobi, z);
    return cudaGetLastError();
}

cudaError_t gate(const FcgScalars* s, cfd2d_fcg_control* ctl, unsigned long long handle, cudaStream_t st) {
    k_gate<<<1, 1, 0, st>>>(s, ctl, (cudaGraphConditionalHandle)handle);
    return cudaGetLastError();
}

cudaError_t zero_rhs(int n, const double* b, double* x, const FcgScalars* s, cudaStream_t st) {
    k_zero_rhs<<<blocks(n), T, 0, st>>>(n, b, x, s);
    return cudaGetLastError();
}

cudaError_t scatter_p(const cfd2d_poisson& op, const double* x, double* p_pad, cudaStream_t st) {
    k_scatter_p<<<blocks((op.nx + 2) * (op.ny + 2)), T, 0, st>>>(op, x, p_pad);
    return cudaGetLastError();
}

}  // namespace fcg
}  // namespace cfd
