// pcg.cu - Jacobi-preconditioned CG for the pressure Poisson equation on the
// fluid cells of the MAC grid, in the iteration form of scipy.sparse.linalg.cg
// (scipy 1.18.1, _isolve/iterative.py:311-431, called by cfd2d/pressure.py:171).
//
// Design (sm_100a): one thread-block cluster of C CTAs (C <= 16) holds the whole
// solver state in shared memory: CTA r owns a slab of interior rows and keeps
// x, r, p (two buffers), 1/diag, diag and the coupling bits of its cells on
// chip for the whole solve. The 5-point operator is applied matrix-free; the
// p values of the two neighbouring rows owned by other CTAs are read through
// distributed shared memory. Each iteration needs exactly two cluster-wide
// reductions (p.q, then r.r and r.z together); partial sums travel through
// DSMEM and every CTA adds the C partials in rank order, so all CTAs see the
// same value and take the same branch. Nothing spins: the only inter-CTA
// waits are hardware cluster barriers, which every CTA reaches the same number
// of times.
//
// Arithmetic order follows the reference: each row of A x is summed in
// increasing column order (scipy's csc_matvec), p = beta*p + z, x += alpha*p,
// r -= alpha*q, the stop test ||r|| < rtol*||b|| at the top of an iteration.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "device.cuh"
#include "pcg.cuh"

namespace cg = cooperative_groups;

namespace cfd {

namespace {

constexpr int kPcgThreads = 512;
constexpr int kSlot = 4 + CFD2D_MAX_COMPONENTS;  // doubles per CTA partial (grid kernel)
constexpr int kMaxCtasPerSm = 32;  // resident CTAs an SM can hold (compute capability 10.0)
constexpr int kArrays = 7;                       // X, R, P0, P1, DI, DG, Z per cell
constexpr int kMaxK = 4;                         // values per cluster reduction

__device__ __forceinline__ int owner_of(int i, int nx, int C) {
    return (int)(((long long)(i + 1) * C - 1) / nx);
}
__device__ __forceinline__ int row0_of(int r, int nx, int C) {
    return (int)((long long)r * nx / C);
}

// Ordered row sum of A x (csc_matvec order). Terms are 0 where no coupling exists.
__device__ __forceinline__ double row_sum(bool periodic, int i, int nx, double tW, double tS,
                                          double tC, double tN, double tE) {
    if (periodic && i == 0) return (((tS + tC) + tN) + tE) + tW;
    if (periodic && i == nx - 1) return (((tE + tW) + tS) + tC) + tN;
    return (((tW + tS) + tC) + tN) + tE;
}

// Cluster-wide sum of K per-thread values. Block tree first: warp sums, then the
// 16 warp partials combined by a 16-lane butterfly in warp 0, whose lane 0 stores
// the CTA partial in this CTA's own slot. After the cluster barrier lanes 0..C-1 of
// warp 0 each load one CTA's partial through DSMEM and a second butterfly adds
// them; lane 0 leaves the sum in shared memory for the whole CTA. Every CTA adds
// the same C values in the same lane positions, so all threads of all CTAs get the
// same bits. Only local stores precede the barrier (remote stores there would
// lengthen it); consecutive reductions alternate slot buffers, so a CTA rewrites a
// slot only after the next barrier, which every reader passes after reading.
template <int K>
__device__ __forceinline__ void cluster_sum(cg::cluster_group& cluster, double (&v)[K],
                                            double* red_smem, double* slots, int C, int me) {
    static_assert(kPcgThreads == 512, "16 warps: the block stage is a 16-lane butterfly");
    (void)me;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) red_smem[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
        double x[K];
#pragma unroll
        for (int k = 0; k < K; ++k) x[k] = (lane < 16) ? red_smem[k * 32 + lane] : 0.0;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
#pragma unroll
            for (int k = 0; k < K; ++k) x[k] += __shfl_xor_sync(0xffffffffu, x[k], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) slots[k] = x[k];
        }
    }
    cluster.sync();
    // the result slots sit above the block-stage slots (k * 32 + w < 3 * 32 + 16)
    double* result = red_smem + 32 * kMaxK - kMaxK;
    if (w == 0) {
        double y[K];
        const double* src = cluster.map_shared_rank(slots, lane < C ? lane : 0);
#pragma unroll
        for (int k = 0; k < K; ++k) y[k] = (lane < C) ? src[k] : 0.0;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
#pragma unroll
            for (int k = 0; k < K; ++k) y[k] += __shfl_xor_sync(0xffffffffu, y[k], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) result[k] = y[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = result[k];
}

}  // namespace

// Off-diagonal entries -(b dx2), -(b dy2) of row (i, j) of the variable-coefficient
// operator (cfd2d/pressure.py:199-216); the west face of column 0 is the periodic face nx
__device__ __forceinline__ void var_coef(const cfd2d_poisson& op, int i, int j, double& w, double& e, double& s,
                                         double& n) {
    const int nx = op.nx, ny = op.ny;
    w = -(op.bx[(size_t)((i == 0) ? nx : i) * (ny + 2) + j + 1] * op.dx2);
    e = -(op.bx[(size_t)(i + 1) * (ny + 2) + j + 1] * op.dx2);
    s = -(op.by[(size_t)(i + 1) * (ny + 1) + j] * op.dy2);
    n = -(op.by[(size_t)(i + 1) * (ny + 1) + j + 1] * op.dy2);
}

template <int CPT, bool PAIR, bool VAR>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg_cluster(PcgLaunch L) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int me = (int)cluster.block_rank();
    if (L.active && *L.active == 0) return;  // uniform over the cluster

    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int r0 = row0_of(me, nx, C), r1 = row0_of(me + 1, nx, C);
    const int rows = r1 - r0;
    const int nloc = rows * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    const int goff = r0 * ny;  // global index of local cell 0

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* R = X + cap;
    double* P0 = R + cap;
    double* P1 = P0 + cap;
    double* DI = P1 + cap;
    double* DG = DI + cap;
    double* Z = DG + cap;
    // variable coefficients (VAR): the four off-diagonal entries of every row
    double* KW = Z + cap;
    double* KE = KW + cap;
    double* KS = KE + cap;
    double* KN = KS + cap;
    uint8_t* NB = reinterpret_cast<uint8_t*>(Z + cap + (VAR ? 4 * cap : 0));
    __shared__ double red_smem[32 * kMaxK];
    __shared__ double slotsA[16 * kMaxK];
    __shared__ double slotsB[16 * kMaxK];
    __shared__ double cmean[CFD2D_MAX_COMPONENTS];
    // consecutive reductions alternate between the two slot buffers, so a buffer is
    // rewritten only after the barrier of the reduction in between, which every CTA
    // reaches after reading it
    int nred = 0;
#define SLOTS() ((nred++ & 1) ? slotsB : slotsA)

    // c / ny by multiply-high: exact for c * ny < 2^32
    const unsigned magic = (unsigned)(((1ull << 32) + (unsigned)ny - 1) / (unsigned)ny);
    // halo rows owned by other CTAs (or by this one when periodic wraps onto itself):
    // generic pointers to their X entries at j = 0; the other arrays follow at
    // multiples of cap, identically in every CTA
    const double* baseW = nullptr;
    const double* baseE = nullptr;
    {
        const int iw = (r0 == 0) ? (periodic ? nx - 1 : -1) : r0 - 1;
        const int ie = (r1 == nx) ? (periodic ? 0 : -1) : r1;
        if (iw >= 0) {
            const int o = owner_of(iw, nx, C);
            baseW = cluster.map_shared_rank(X, o) + (iw - row0_of(o, nx, C)) * ny;
        }
        if (ie >= 0) {
            const int o = owner_of(ie, nx, C);
            baseE = cluster.map_shared_rank(X, o) + (ie - row0_of(o, nx, C)) * ny;
        }
    }

    // ------------------------------------------------------------ prologue
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double nzx = 0.0;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int gidx = goff + c;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        const double x0 = op.x0[gidx];
        X[c] = x0;
        DI[c] = op.dinv[gidx];
        DG[c] = op.diag[gidx];
        if constexpr (VAR) {
            const int li = (int)__umulhi((unsigned)c, magic);
            var_coef(op, r0 + li, c - li * ny, KW[c], KE[c], KS[c], KN[c]);
        }
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                // div(F, G) / dt at interior cell (i+1, j+1) (cfd2d/solver.py:264-266)
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                const int pu = ny + 2, pv = ny + 1;
                const int ig = r0 + li + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            if (x0 != 0.0) nzx += 1.0;
        }
        R[c] = braw;
    }
    // scipy computes A x0 only if x0 has a nonzero (iterative.py: "if x.any()")
    {
        double v[1] = {nzx};
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        nzx = v[0];
    }
    const bool x_any = nzx > 0.0;
    // Neumann-component means of b (cfd2d/pressure.py:155-160), one reduction each
    const int ncomp = op.ncomp;
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += R[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();

    // b = -(b_raw - mean), r = b - A x0, z = M^-1 r, norms
    double part[3] = {0.0, 0.0, 0.0};
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const uint8_t nb = NB[c];
        if (!(nb & 0x80)) { P1[c] = 0.0; P0[c] = 0.0; R[c] = 0.0; Z[c] = 0.0; continue; }
        double b = R[c];
        if (ncomp > 0) {
            const int lab = op.label[goff + c];
            if (lab >= 0) b = b - cmean[lab];
        }
        b = -b;
        P1[c] = b;  // kept for the ||b|| == 0 return
        double r = b;
        if (x_any) {
            const int li = (int)__umulhi((unsigned)c, magic);
            const int j = c - li * ny;
            double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
            const double kS = VAR ? KS[c] : mdy2, kN = VAR ? KN[c] : mdy2;
            const double kW = VAR ? KW[c] : mdx2, kE = VAR ? KE[c] : mdx2;
            if (nb & 2) tS = kS * X[c - 1];
            if (nb & 4) tN = kN * X[c + 1];
            if (nb & 1) tW = kW * ((li > 0) ? X[c - ny] : baseW[j]);
            if (nb & 8) tE = kE * ((li < rows - 1) ? X[c + ny] : baseE[j]);
            r = b - row_sum(periodic, r0 + li, nx, tW, tS, DG[c] * X[c], tN, tE);
        }
        // R and Z are read by other CTAs only inside the loop, after the barrier of
        // the reduction below; X (read here across CTAs) is unchanged until then
        R[c] = r;
        P0[c] = 0.0;
        const double z = DI[c] * r;
        Z[c] = z;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * z;
    }
    cluster_sum<3>(cluster, part, red_smem, SLOTS(), C, me);
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];  // r . z for the first iteration
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;
    if (bnrm2 == 0.0) {
        // scipy returns b itself
        for (int c = tid; c < nloc; c += kPcgThreads) X[c] = P1[c];
        converged = true;
    } else {
        double beta = 0.0;
        int cur = 0;  // p of this iteration goes to buffer cur (P0 or P1)
        double q[PAIR ? 2 * CPT : CPT];
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            double* Pn = cur ? P1 : P0;
            const double* Po = cur ? P0 : P1;
            const int po = cur ? 2 * cap : 3 * cap;  // offset of the previous p from X
            const bool first = (it == 0);
            double pq = 0.0;
            if constexpr (PAIR) {
                // two cells (c, c+1) of one row per slot; ny is even, so c is even and
                // every 16-byte pair load is aligned
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    q[2 * k] = 0.0;
                    q[2 * k + 1] = 0.0;
                    const int c = 2 * (tid + k * kPcgThreads);
                    if (c >= nloc) continue;
                    const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                    const unsigned nb0 = nb2 & 0xFFu, nb1 = nb2 >> 8;
                    if (!((nb0 | nb1) & 0x80u)) continue;
                    const int li = (int)__umulhi((unsigned)c, magic);
                    const int j = c - li * ny;
                    const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                    double pC0 = z2.x, pC1 = z2.y;
                    if (!first) {
                        const double2 o2 = *reinterpret_cast<const double2*>(Po + c);
                        pC0 = o2.x * beta + z2.x;
                        pC1 = o2.y * beta + z2.y;
                    }
                    // solid cells carry p = z = 0 and no coupling bits, so their terms vanish
                    double kS0 = mdy2, kS1 = mdy2, kN0 = mdy2, kN1 = mdy2;
                    double kW0 = mdx2, kW1 = mdx2, kE0 = mdx2, kE1 = mdx2;
                    if constexpr (VAR) {
                        const double2 ks = *reinterpret_cast<const double2*>(KS + c);
                        const double2 kn = *reinterpret_cast<const double2*>(KN + c);
                        const double2 kw = *reinterpret_cast<const double2*>(KW + c);
                        const double2 ke = *reinterpret_cast<const double2*>(KE + c);
                        kS0 = ks.x; kS1 = ks.y; kN0 = kn.x; kN1 = kn.y;
                        kW0 = kw.x; kW1 = kw.y; kE0 = ke.x; kE1 = ke.y;
                    }
                    double tW0 = 0.0, tW1 = 0.0, tE0 = 0.0, tE1 = 0.0;
                    const double tS0 = (nb0 & 2) ? kS0 * (first ? Z[c - 1] : Po[c - 1] * beta + Z[c - 1]) : 0.0;
                    const double tN0 = (nb0 & 4) ? kN0 * pC1 : 0.0;
                    const double tS1 = (nb1 & 2) ? kS1 * pC0 : 0.0;
                    const double tN1 = (nb1 & 4) ? kN1 * (first ? Z[c + 2] : Po[c + 2] * beta + Z[c + 2]) : 0.0;
                    if ((nb0 | nb1) & 1) {
                        const double* g = (li > 0) ? (X + c - ny) : (baseW + j);
                        const double2 gz = *reinterpret_cast<const double2*>(g + 6 * cap);
                        double w0 = gz.x, w1 = gz.y;
                        if (!first) {
                            const double2 go = *reinterpret_cast<const double2*>(g + po);
                            w0 = go.x * beta + gz.x;
                            w1 = go.y * beta + gz.y;
                        }
                        if (nb0 & 1) tW0 = kW0 * w0;
                        if (nb1 & 1) tW1 = kW1 * w1;
                    }
                    if ((nb0 | nb1) & 8) {
                        const double* g = (li < rows - 1) ? (X + c + ny) : (baseE + j);
                        const double2 gz = *reinterpret_cast<const double2*>(g + 6 * cap);
                        double e0 = gz.x, e1 = gz.y;
                        if (!first) {
                            const double2 go = *reinterpret_cast<const double2*>(g + po);
                            e0 = go.x * beta + gz.x;
                            e1 = go.y * beta + gz.y;
                        }
                        if (nb0 & 8) tE0 = kE0 * e0;
                        if (nb1 & 8) tE1 = kE1 * e1;
                    }
                    const double2 dg = *reinterpret_cast<const double2*>(DG + c);
                    const int i = r0 + li;
                    const double q0 = row_sum(periodic, i, nx, tW0, tS0, dg.x * pC0, tN0, tE0);
                    const double q1 = row_sum(periodic, i, nx, tW1, tS1, dg.y * pC1, tN1, tE1);
                    *reinterpret_cast<double2*>(Pn + c) = make_double2(pC0, pC1);
                    q[2 * k] = q0;
                    q[2 * k + 1] = q1;
                    pq += pC0 * q0;
                    pq += pC1 * q1;
                }
            } else {
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                q[k] = 0.0;
                const int c = tid + k * kPcgThreads;
                if (c >= nloc) continue;
                const uint8_t nb = NB[c];
                if (!(nb & 0x80)) continue;
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                // p_new = beta * p_old + z, recomputed for the neighbours from their
                // previous p and z instead of waiting for their owners
                const double pC = first ? Z[c] : Po[c] * beta + Z[c];
                const double kS = VAR ? KS[c] : mdy2, kN = VAR ? KN[c] : mdy2;
                const double kW = VAR ? KW[c] : mdx2, kE = VAR ? KE[c] : mdx2;
                double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
                if (nb & 2) tS = kS * (first ? Z[c - 1] : Po[c - 1] * beta + Z[c - 1]);
                if (nb & 4) tN = kN * (first ? Z[c + 1] : Po[c + 1] * beta + Z[c + 1]);
                if (nb & 1) {
                    const double* g = (li > 0) ? (X + c - ny) : (baseW + j);
                    tW = kW * (first ? g[6 * cap] : g[po] * beta + g[6 * cap]);
                }
                if (nb & 8) {
                    const double* g = (li < rows - 1) ? (X + c + ny) : (baseE + j);
                    tE = kE * (first ? g[6 * cap] : g[po] * beta + g[6 * cap]);
                }
                const double qq = row_sum(periodic, r0 + li, nx, tW, tS, DG[c] * pC, tN, tE);
                Pn[c] = pC;
                q[k] = qq;
                pq += pC * qq;
            }
            }
            {
                double v[1] = {pq};
                cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
                pq = v[0];
            }
            const double alpha = rho / pq;
            double v2[2] = {0.0, 0.0};
            if constexpr (PAIR) {
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const int c = 2 * (tid + k * kPcgThreads);
                    if (c >= nloc) continue;
                    const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                    const bool f0 = nb2 & 0x80u, f1 = (nb2 >> 8) & 0x80u;
                    if (!(f0 || f1)) continue;
                    double2 x2 = *reinterpret_cast<const double2*>(X + c);
                    double2 r2 = *reinterpret_cast<const double2*>(R + c);
                    double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                    const double2 p2 = *reinterpret_cast<const double2*>(Pn + c);
                    const double2 d2 = *reinterpret_cast<const double2*>(DI + c);
                    if (f0) {
                        x2.x = x2.x + alpha * p2.x;
                        r2.x = r2.x - alpha * q[2 * k];
                        z2.x = d2.x * r2.x;
                        v2[0] += r2.x * r2.x;
                        v2[1] += r2.x * z2.x;
                    }
                    if (f1) {
                        x2.y = x2.y + alpha * p2.y;
                        r2.y = r2.y - alpha * q[2 * k + 1];
                        z2.y = d2.y * r2.y;
                        v2[0] += r2.y * r2.y;
                        v2[1] += r2.y * z2.y;
                    }
                    *reinterpret_cast<double2*>(X + c) = x2;
                    *reinterpret_cast<double2*>(R + c) = r2;
                    *reinterpret_cast<double2*>(Z + c) = z2;
                }
            } else {
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = tid + k * kPcgThreads;
                if (c >= nloc) continue;
                if (!(NB[c] & 0x80)) continue;
                X[c] = X[c] + alpha * Pn[c];
                const double r = R[c] - alpha * q[k];
                R[c] = r;
                const double z = DI[c] * r;
                Z[c] = z;
                v2[0] += r * r;
                v2[1] += r * z;
            }
            }
            cluster_sum<2>(cluster, v2, red_smem, SLOTS(), C, me);
            rr = v2[0];
            beta = v2[1] / rho;
            rho = v2[1];
            cur ^= 1;
        }
    }
    // ------------------------------------------------------------ epilogue
    __syncthreads();
    for (int c = tid; c < nloc; c += kPcgThreads) op.x0[goff + c] = X[c];
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += X[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int li = (int)__umulhi((unsigned)c, magic);
        const int j = c - li * ny;
        const int i = r0 + li;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) pv = pv - cmean[lab];
            }
        }
        if (!L.p_padded) {
            L.p_out[goff + c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            // periodic ghost rows: p[0,:] = p[nx,:], p[nx+1,:] = p[1,:]
            if (periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
        }
    }
    if (L.p_padded) {
        // ghost entries j = 0, ny + 1 of own rows, and the outer ghost rows
        for (int i = r0 + tid; i < r1; i += kPcgThreads) {
            L.p_out[(i + 1) * pp] = 0.0;
            L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
        if (me == 0) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
        }
        if (me == C - 1) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
    // keep every CTA's shared memory alive until all remote readers are done
    cluster.sync();
#undef SLOTS
}

// ---------------------------------------------------------------- single-reduction cluster form
// The on-chip cluster solver with the Jacobi-PCG recurrence of Chronopoulos and Gear
// (the slab solver's k_pcg_slab1 recurrence): one cluster barrier per iteration, the
// reduction of r.z, z.w and r.r together. Even ny and constant coefficients (cell
// pairs, as k_pcg_cluster<CPT, true, false>). Each iteration updates p = z + beta p,
// q = w + beta q (= A p), x, r and z = D^-1 r of the CTA's own cells, then needs the
// new z of the two halo rows for w = A z. Instead of a second barrier, every CTA has
// exported the (r, q, w) of its first and last row before the previous reduction's
// barrier, into one of two buffers by iteration parity, and each neighbour recomputes
// the halo row's new z from them with the owner's own operations (the same bits). A
// buffer is rewritten two iterations later, after a barrier that every reader passes
// once done with it. Shared memory per CTA: the cluster layout plus 2 x 3 x 2 export
// rows and the two halo rows of z (14 ny doubles). Selected by grid_ctas = -2 on the
// grids the cluster solver takes.
constexpr int kExportRows = 12;  // 2 parities x (r, q, w) x (first row, last row)
constexpr int kHaloPer = 2;      // halo cells per thread: 2 ny <= 2 x 512

inline size_t smem_bytes1(int cap, int ny) {
    return (size_t)cap * (kArrays * sizeof(double) + 1) + (size_t)(kExportRows + 2) * ny * sizeof(double) + 16;
}

template <int CPT>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg_cluster1(PcgLaunch L) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int me = (int)cluster.block_rank();
    if (L.active && *L.active == 0) return;  // uniform over the cluster

    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int r0 = row0_of(me, nx, C), r1 = row0_of(me + 1, nx, C);
    const int rows = r1 - r0;
    const int nloc = rows * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    const int goff = r0 * ny;

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* R = X + cap;
    double* P = R + cap;  // p
    double* Q = P + cap;  // q = A p
    double* DI = Q + cap;
    double* DG = DI + cap;
    double* Z = DG + cap;
    double* EX = Z + cap;                       // [parity][r, q, w][first, last row][ny]
    double* HZ = EX + (size_t)kExportRows * ny;  // new z of the west halo row at [0, ny), east at [ny, 2 ny)
    uint8_t* NB = reinterpret_cast<uint8_t*>(HZ + 2 * ny);
    __shared__ double red_smem[32 * kMaxK];
    __shared__ double slotsA[16 * kMaxK];
    __shared__ double slotsB[16 * kMaxK];
    __shared__ double cmean[CFD2D_MAX_COMPONENTS];
    int nred = 0;
#define SLOTS() ((nred++ & 1) ? slotsB : slotsA)
    const unsigned magic = (unsigned)(((1ull << 32) + (unsigned)ny - 1) / (unsigned)ny);

    // halo rows: the west one is its owner's last row (export side 1), the east one its
    // owner's first row (side 0). hb: the owner's shared memory (its X); ho: the halo
    // row's first cell in the owner's numbering. The layout is the same in every CTA.
    const int iw = (r0 == 0) ? (periodic ? nx - 1 : -1) : r0 - 1;
    const int ie = (r1 == nx) ? (periodic ? 0 : -1) : r1;
    const double* hbW = nullptr;
    const double* hbE = nullptr;
    int hoW = 0, hoE = 0;
    if (iw >= 0) {
        const int o = owner_of(iw, nx, C);
        hbW = cluster.map_shared_rank(X, o);
        hoW = (iw - row0_of(o, nx, C)) * ny;
    }
    if (ie >= 0) {
        const int o = owner_of(ie, nx, C);
        hbE = cluster.map_shared_rank(X, o);
        hoE = (ie - row0_of(o, nx, C)) * ny;
    }
    const size_t exOff = (size_t)kArrays * cap;                               // EX from X
    const size_t nbOff = ((size_t)kArrays * cap + (size_t)(kExportRows + 2) * ny) * sizeof(double);  // NB, bytes

    // ------------------------------------------------------------ prologue
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double nzx = 0.0;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int gidx = goff + c;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        const double x0 = op.x0[gidx];
        X[c] = x0;
        DI[c] = op.dinv[gidx];
        DG[c] = op.diag[gidx];
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                // div(F, G) / dt at interior cell (i+1, j+1) (cfd2d/solver.py:264-266)
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                const int pu = ny + 2, pv = ny + 1;
                const int ig = r0 + li + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            if (x0 != 0.0) nzx += 1.0;
        }
        R[c] = braw;
    }
    {
        double v[1] = {nzx};
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        nzx = v[0];
    }
    const bool x_any = nzx > 0.0;
    const int ncomp = op.ncomp;
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += R[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();
    double part[3] = {0.0, 0.0, 0.0};
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const uint8_t nb = NB[c];
        if (!(nb & 0x80)) { P[c] = 0.0; Q[c] = 0.0; R[c] = 0.0; Z[c] = 0.0; continue; }
        double b = R[c];
        if (ncomp > 0) {
            const int lab = op.label[goff + c];
            if (lab >= 0) b = b - cmean[lab];
        }
        b = -b;
        P[c] = b;  // kept for the ||b|| == 0 return
        double r = b;
        if (x_any) {
            const int li = (int)__umulhi((unsigned)c, magic);
            const int j = c - li * ny;
            double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
            if (nb & 2) tS = mdy2 * X[c - 1];
            if (nb & 4) tN = mdy2 * X[c + 1];
            if (nb & 1) tW = mdx2 * ((li > 0) ? X[c - ny] : hbW[hoW + j]);
            if (nb & 8) tE = mdx2 * ((li < rows - 1) ? X[c + ny] : hbE[hoE + j]);
            r = b - row_sum(periodic, r0 + li, nx, tW, tS, DG[c] * X[c], tN, tE);
        }
        // R and Z are read by other CTAs only after the barrier of the reduction below;
        // X (read here across CTAs) is unchanged until then
        R[c] = r;
        Q[c] = 0.0;
        const double z = DI[c] * r;
        Z[c] = z;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * z;
    }
    cluster_sum<3>(cluster, part, red_smem, SLOTS(), C, me);
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;

    // w = A z of a cell pair (c, c + 1); the halo rows' z from HZ
    auto az_pair = [&](int c, int li, double& w0, double& w1) {
        const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
        const unsigned nb0 = nb2 & 0xFFu, nb1 = nb2 >> 8;
        w0 = 0.0;
        w1 = 0.0;
        if (!((nb0 | nb1) & 0x80u)) return;
        const int j = c - li * ny;
        const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
        double tW0 = 0.0, tW1 = 0.0, tE0 = 0.0, tE1 = 0.0;
        const double tS0 = (nb0 & 2) ? mdy2 * Z[c - 1] : 0.0;
        const double tN0 = (nb0 & 4) ? mdy2 * z2.y : 0.0;
        const double tS1 = (nb1 & 2) ? mdy2 * z2.x : 0.0;
        const double tN1 = (nb1 & 4) ? mdy2 * Z[c + 2] : 0.0;
        if ((nb0 | nb1) & 1) {
            const double2 g = *reinterpret_cast<const double2*>(li > 0 ? (Z + c - ny) : (HZ + j));
            if (nb0 & 1) tW0 = mdx2 * g.x;
            if (nb1 & 1) tW1 = mdx2 * g.y;
        }
        if ((nb0 | nb1) & 8) {
            const double2 g = *reinterpret_cast<const double2*>(li < rows - 1 ? (Z + c + ny) : (HZ + ny + j));
            if (nb0 & 8) tE0 = mdx2 * g.x;
            if (nb1 & 8) tE1 = mdx2 * g.y;
        }
        const double2 dg = *reinterpret_cast<const double2*>(DG + c);
        const int i = r0 + li;
        w0 = row_sum(periodic, i, nx, tW0, tS0, dg.x * z2.x, tN0, tE0);
        w1 = row_sum(periodic, i, nx, tW1, tS1, dg.y * z2.y, tN1, tE1);
    };
    double w[2 * CPT];
    // w of every own pair and its z.w partial
    auto apply_w = [&]() -> double {
        double d = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int c = 2 * (tid + k * kPcgThreads);
            if (c >= nloc) { w[2 * k] = w[2 * k + 1] = 0.0; continue; }
            const int li = (int)__umulhi((unsigned)c, magic);
            az_pair(c, li, w[2 * k], w[2 * k + 1]);
            const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
            d += z2.x * w[2 * k];
            d += z2.y * w[2 * k + 1];
        }
        return d;
    };
    // this CTA's first and last row of (r, q, w) into export buffer par
    auto export_rows = [&](int par) {
        double* ex = EX + (size_t)par * 6 * ny;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int c = 2 * (tid + k * kPcgThreads);
            if (c >= nloc) continue;
            const int li = (int)__umulhi((unsigned)c, magic);
            const int j = c - li * ny;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                if (li != (side == 0 ? 0 : rows - 1)) continue;
                *reinterpret_cast<double2*>(ex + (0 * 2 + side) * ny + j) = *reinterpret_cast<const double2*>(R + c);
                *reinterpret_cast<double2*>(ex + (1 * 2 + side) * ny + j) = *reinterpret_cast<const double2*>(Q + c);
                *reinterpret_cast<double2*>(ex + (2 * 2 + side) * ny + j) = make_double2(w[2 * k], w[2 * k + 1]);
            }
        }
    };
    // the halo rows' new z from their owners' export buffer par, with the owner's own
    // operations: q = w (first iteration) or q beta + w, r - alpha q, D^-1 r on fluid
    // cells. The loads (coupling bits, r, q, w, 1/diag; all in bounds, taken whether or
    // not the cell is fluid) are issued at the start of the iteration into registers,
    // so their latency passes under the update of the CTA's own cells; halo_store
    // forms z and writes HZ afterwards. Thread t takes halo cells t, t + 512, ... (2 ny
    // <= kHaloPer x 512).
    double hr[kHaloPer], hq[kHaloPer], hw[kHaloPer], hd[kHaloPer];
    uint8_t hn[kHaloPer];
    auto halo_load = [&](int par) {
#pragma unroll
        for (int u = 0; u < kHaloPer; ++u) {
            const int t = tid + u * kPcgThreads;
            hn[u] = 0;
            if (t >= 2 * ny) continue;
            const bool west = t < ny;
            const int j = west ? t : t - ny;
            const double* hb = west ? hbW : hbE;
            if (!hb) continue;
            const int cell = (west ? hoW : hoE) + j;
            const double* ex = hb + exOff + (size_t)par * 6 * ny + (west ? ny : 0) + j;
            hn[u] = reinterpret_cast<const uint8_t*>(hb)[nbOff + cell];
            hr[u] = ex[0];
            hq[u] = ex[2 * ny];
            hw[u] = ex[4 * ny];
            hd[u] = hb[4 * (size_t)cap + cell];
        }
    };
    auto halo_store = [&](bool first, double alpha, double beta) {
#pragma unroll
        for (int u = 0; u < kHaloPer; ++u) {
            const int t = tid + u * kPcgThreads;
            if (t >= 2 * ny) continue;
            double z = 0.0;
            if (hn[u] & 0x80) {
                const double qn = first ? hw[u] : hq[u] * beta + hw[u];
                const double rn = hr[u] - alpha * qn;
                z = hd[u] * rn;
            }
            HZ[t] = z;
        }
    };

    // w = A z and delta = z.w of the initial z: the reduction above made every CTA's z
    // final, so the halo rows are read from their owners directly
    double delta;
    for (int t = tid; t < 2 * ny; t += kPcgThreads) {
        const bool west = t < ny;
        const double* hb = west ? hbW : hbE;
        HZ[t] = hb ? hb[6 * (size_t)cap + (west ? hoW : hoE) + (west ? t : t - ny)] : 0.0;
    }
    __syncthreads();
    {
        double d[1] = {apply_w()};
        export_rows(0);
        cluster_sum<1>(cluster, d, red_smem, SLOTS(), C, me);
        delta = d[0];
    }
    if (bnrm2 == 0.0) {
        // scipy returns b itself
        for (int c = tid; c < nloc; c += kPcgThreads) X[c] = P[c];
        converged = true;
    } else {
        double rho_prev = 1.0, alpha_prev = 1.0;
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            const bool first = (it == 0);
            double beta = 0.0, pq = delta;
            if (!first) {
                beta = rho / rho_prev;
                pq = delta - (beta * rho) / alpha_prev;
            }
            const double alpha = rho / pq;
            halo_load(it & 1);
            double v3[3] = {0.0, 0.0, 0.0};  // r.z, z.w, r.r
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = 2 * (tid + k * kPcgThreads);
                if (c >= nloc) continue;
                const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                const bool f0 = nb2 & 0x80u, f1 = (nb2 >> 8) & 0x80u;
                if (!(f0 || f1)) continue;
                double2 x2 = *reinterpret_cast<const double2*>(X + c);
                double2 r2 = *reinterpret_cast<const double2*>(R + c);
                double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                double2 p2 = *reinterpret_cast<const double2*>(P + c);
                double2 q2 = *reinterpret_cast<const double2*>(Q + c);
                const double2 d2 = *reinterpret_cast<const double2*>(DI + c);
                if (first) {
                    p2 = z2;
                    q2 = make_double2(w[2 * k], w[2 * k + 1]);
                } else {
                    p2 = make_double2(p2.x * beta + z2.x, p2.y * beta + z2.y);
                    q2 = make_double2(q2.x * beta + w[2 * k], q2.y * beta + w[2 * k + 1]);
                }
                if (f0) {
                    x2.x = x2.x + alpha * p2.x;
                    r2.x = r2.x - alpha * q2.x;
                    z2.x = d2.x * r2.x;
                    v3[0] += r2.x * z2.x;
                    v3[2] += r2.x * r2.x;
                }
                if (f1) {
                    x2.y = x2.y + alpha * p2.y;
                    r2.y = r2.y - alpha * q2.y;
                    z2.y = d2.y * r2.y;
                    v3[0] += r2.y * z2.y;
                    v3[2] += r2.y * r2.y;
                }
                *reinterpret_cast<double2*>(X + c) = x2;
                *reinterpret_cast<double2*>(R + c) = r2;
                *reinterpret_cast<double2*>(Z + c) = z2;
                *reinterpret_cast<double2*>(P + c) = p2;
                *reinterpret_cast<double2*>(Q + c) = q2;
            }
            halo_store(first, alpha, beta);
            __syncthreads();
            v3[1] = apply_w();
            export_rows((it + 1) & 1);
            cluster_sum<3>(cluster, v3, red_smem, SLOTS(), C, me);
            rho_prev = rho;
            alpha_prev = alpha;
            rho = v3[0];
            delta = v3[1];
            rr = v3[2];
        }
    }
    // ------------------------------------------------------------ epilogue
    __syncthreads();
    for (int c = tid; c < nloc; c += kPcgThreads) op.x0[goff + c] = X[c];
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += X[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int li = (int)__umulhi((unsigned)c, magic);
        const int j = c - li * ny;
        const int i = r0 + li;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) pv = pv - cmean[lab];
            }
        }
        if (!L.p_padded) {
            L.p_out[goff + c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            if (periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
        }
    }
    if (L.p_padded) {
        for (int i = r0 + tid; i < r1; i += kPcgThreads) {
            L.p_out[(i + 1) * pp] = 0.0;
            L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
        if (me == 0) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
        }
        if (me == C - 1) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
    // keep every CTA's shared memory alive until all remote readers are done
    cluster.sync();
#undef SLOTS
}

// ---------------------------------------------------------------- mixed precision
// Ordered row sum in FP32 (the inner iterations of the mixed solver).
__device__ __forceinline__ float row_sum_f(bool periodic, int i, int nx, float tW, float tS, float tC, float tN,
                                           float tE) {
    if (periodic && i == 0) return (((tS + tC) + tN) + tE) + tW;
    if (periodic && i == nx - 1) return (((tE + tW) + tS) + tC) + tN;
    return (((tW + tS) + tC) + tN) + tE;
}

// Jacobi-PCG with FP32 iterations and FP64 iterative refinement, cluster-resident
// (an upgrade beside the scipy-form solver above; no reference counterpart).
// Outer loop in FP64: r = b - A x, stop when ||r|| < rtol ||b||; otherwise an FP32
// Jacobi-PCG solves A d = r from d = 0 until its recursive residual falls below
// kInnerTol ||r||, and x += d in FP64. Every dot product is accumulated and reduced
// in FP64. Shared memory per cell: x and b in FP64, d, r, p (two buffers), z,
// 1/diag and diag in FP32, the coupling bits: 45 bytes.
constexpr float kInnerTol = 1e-4f;

template <int CPT>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg_cluster_mixed(PcgLaunch L) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int me = (int)cluster.block_rank();
    if (L.active && *L.active == 0) return;  // uniform over the cluster

    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int r0 = row0_of(me, nx, C), r1 = row0_of(me + 1, nx, C);
    const int rows = r1 - r0;
    const int nloc = rows * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    const float fdx2 = (float)mdx2, fdy2 = (float)mdy2;
    const int goff = r0 * ny;

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* B = X + cap;
    float* D = reinterpret_cast<float*>(B + cap);
    float* R = D + cap;
    float* P0 = R + cap;
    float* P1 = P0 + cap;
    float* Z = P1 + cap;
    float* DI = Z + cap;
    float* DG = DI + cap;
    uint8_t* NB = reinterpret_cast<uint8_t*>(DG + cap);
    __shared__ double red_smem[32 * kMaxK];
    __shared__ double slotsA[16 * kMaxK];
    __shared__ double slotsB[16 * kMaxK];
    __shared__ double cmean[CFD2D_MAX_COMPONENTS];
    int nred = 0;
#define SLOTS() ((nred++ & 1) ? slotsB : slotsA)

    const unsigned magic = (unsigned)(((1ull << 32) + (unsigned)ny - 1) / (unsigned)ny);
    // neighbouring rows in other CTAs: their x (FP64) and their FP32 arrays at j = 0
    const double* baseWx = nullptr;
    const double* baseEx = nullptr;
    const float* baseWf = nullptr;
    const float* baseEf = nullptr;
    {
        const int iw = (r0 == 0) ? (periodic ? nx - 1 : -1) : r0 - 1;
        const int ie = (r1 == nx) ? (periodic ? 0 : -1) : r1;
        if (iw >= 0) {
            const int o = owner_of(iw, nx, C);
            const int off = (iw - row0_of(o, nx, C)) * ny;
            baseWx = cluster.map_shared_rank(X, o) + off;
            baseWf = cluster.map_shared_rank(D, o) + off;
        }
        if (ie >= 0) {
            const int o = owner_of(ie, nx, C);
            const int off = (ie - row0_of(o, nx, C)) * ny;
            baseEx = cluster.map_shared_rank(X, o) + off;
            baseEf = cluster.map_shared_rank(D, o) + off;
        }
    }

    // ------------------------------------------------------------ prologue
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int gidx = goff + c;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        X[c] = op.x0[gidx];
        DI[c] = (float)op.dinv[gidx];
        DG[c] = (float)op.diag[gidx];
        P0[c] = 0.0f;
        P1[c] = 0.0f;
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                const int pu = ny + 2, pv = ny + 1;
                const int ig = r0 + li + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
        }
        B[c] = braw;
    }
    const int ncomp = op.ncomp;
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += B[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();
    double bb = 0.0;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        double b = 0.0;
        if (NB[c] & 0x80) {
            b = B[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) b = b - cmean[lab];
            }
            b = -b;
        }
        B[c] = b;
        bb += b * b;
    }
    {
        // also the barrier after which other CTAs read this CTA's x
        double v[1] = {bb};
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        bb = v[0];
    }
    const double bnrm2 = sqrt(bb);
    const double atol = L.rtol * bnrm2;
    int total = 0;
    bool converged = false;
    if (bnrm2 == 0.0) {
        for (int c = tid; c < nloc; c += kPcgThreads) X[c] = B[c];
        converged = true;
    } else {
        for (int outer = 0; outer < 64 && !converged; ++outer) {
            // true residual in FP64; the inner iteration starts from d = 0
            double part[2] = {0.0, 0.0};
            for (int c = tid; c < nloc; c += kPcgThreads) {
                const uint8_t nb = NB[c];
                D[c] = 0.0f;
                if (!(nb & 0x80)) { R[c] = 0.0f; Z[c] = 0.0f; continue; }
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
                if (nb & 2) tS = mdy2 * X[c - 1];
                if (nb & 4) tN = mdy2 * X[c + 1];
                if (nb & 1) tW = mdx2 * ((li > 0) ? X[c - ny] : baseWx[j]);
                if (nb & 8) tE = mdx2 * ((li < rows - 1) ? X[c + ny] : baseEx[j]);
                const double r = B[c] - row_sum(periodic, r0 + li, nx, tW, tS, op.diag[goff + c] * X[c], tN, tE);
                const float rf = (float)r;
                const float zf = DI[c] * rf;
                R[c] = rf;
                Z[c] = zf;
                part[0] += r * r;
                part[1] += (double)rf * (double)zf;
            }
            cluster_sum<2>(cluster, part, red_smem, SLOTS(), C, me);
            const double rnorm = sqrt(part[0]);
            if (rnorm < atol) { converged = true; break; }
            if (total >= L.maxiter) break;
            // FP32 Jacobi-PCG on A d = r (the p recompute and halo scheme of the FP64 solver)
            const double tol_in = (double)kInnerTol * rnorm;
            double rr = part[0], rho = part[1], beta = 0.0;
            int cur = 0;
            float q[CPT];
            for (int k = 0; total < L.maxiter; ++k, ++total) {
                if (k > 0 && sqrt(rr) < tol_in) break;
                float* Pn = cur ? P1 : P0;
                const float* Po = cur ? P0 : P1;
                const int po = cur ? 2 * cap : 3 * cap;  // previous p from D
                const bool first = (k == 0);
                const float fb = (float)beta;
                double pq = 0.0;
#pragma unroll
                for (int s = 0; s < CPT; ++s) {
                    q[s] = 0.0f;
                    const int c = tid + s * kPcgThreads;
                    if (c >= nloc) continue;
                    const uint8_t nb = NB[c];
                    if (!(nb & 0x80)) continue;
                    const int li = (int)__umulhi((unsigned)c, magic);
                    const int j = c - li * ny;
                    const float pC = first ? Z[c] : Po[c] * fb + Z[c];
                    float tW = 0.0f, tS = 0.0f, tN = 0.0f, tE = 0.0f;
                    if (nb & 2) tS = fdy2 * (first ? Z[c - 1] : Po[c - 1] * fb + Z[c - 1]);
                    if (nb & 4) tN = fdy2 * (first ? Z[c + 1] : Po[c + 1] * fb + Z[c + 1]);
                    if (nb & 1) {
                        const float* g = (li > 0) ? (D + c - ny) : (baseWf + j);
                        tW = fdx2 * (first ? g[4 * cap] : g[po] * fb + g[4 * cap]);
                    }
                    if (nb & 8) {
                        const float* g = (li < rows - 1) ? (D + c + ny) : (baseEf + j);
                        tE = fdx2 * (first ? g[4 * cap] : g[po] * fb + g[4 * cap]);
                    }
                    const float qq = row_sum_f(periodic, r0 + li, nx, tW, tS, DG[c] * pC, tN, tE);
                    Pn[c] = pC;
                    q[s] = qq;
                    pq += (double)pC * (double)qq;
                }
                {
                    double v[1] = {pq};
                    cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
                    pq = v[0];
                }
                const float alpha = (float)(rho / pq);
                double v2[2] = {0.0, 0.0};
#pragma unroll
                for (int s = 0; s < CPT; ++s) {
                    const int c = tid + s * kPcgThreads;
                    if (c >= nloc) continue;
                    if (!(NB[c] & 0x80)) continue;
                    D[c] = D[c] + alpha * Pn[c];
                    const float r = R[c] - alpha * q[s];
                    R[c] = r;
                    const float z = DI[c] * r;
                    Z[c] = z;
                    v2[0] += (double)r * (double)r;
                    v2[1] += (double)r * (double)z;
                }
                cluster_sum<2>(cluster, v2, red_smem, SLOTS(), C, me);
                rr = v2[0];
                beta = v2[1] / rho;
                rho = v2[1];
                cur ^= 1;
            }
            // x += d in FP64; the barrier makes the new x visible to the neighbours'
            // residual rows (and ends every read of this CTA's d, r, z)
            for (int c = tid; c < nloc; c += kPcgThreads)
                if (NB[c] & 0x80) X[c] = X[c] + (double)D[c];
            cluster.sync();
        }
    }
    // ------------------------------------------------------------ epilogue
    __syncthreads();
    for (int c = tid; c < nloc; c += kPcgThreads) op.x0[goff + c] = X[c];
    for (int k = 0; k < ncomp; ++k) {
        double v[1] = {0.0};
        for (int c = tid; c < nloc; c += kPcgThreads)
            if ((NB[c] & 0x80) && op.label[goff + c] == k) v[0] += X[c];
        cluster_sum<1>(cluster, v, red_smem, SLOTS(), C, me);
        if (tid == 0) cmean[k] = v[0] / op.comp_count[k];
    }
    __syncthreads();
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int li = (int)__umulhi((unsigned)c, magic);
        const int j = c - li * ny;
        const int i = r0 + li;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) pv = pv - cmean[lab];
            }
        }
        if (!L.p_padded) {
            L.p_out[goff + c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            if (periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
        }
    }
    if (L.p_padded) {
        for (int i = r0 + tid; i < r1; i += kPcgThreads) {
            L.p_out[(i + 1) * pp] = 0.0;
            L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
        if (me == 0) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
        }
        if (me == C - 1) {
            for (int j = tid; j < pp; j += kPcgThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = total;
        if (L.iters_out2) *L.iters_out2 = total;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
    cluster.sync();
#undef SLOTS
}

// ---------------------------------------------------------------- grid-persistent variant
// For grids beyond the on-chip capacity of one cluster: a cooperative launch of
// G co-resident CTAs over all SMs, vectors in global memory (the workspace),
// the same iteration form and operation order. CTA b owns a contiguous range of
// cells. p_new of a cell's neighbours is recomputed from r, p_old and 1/diag
// (as in the cluster kernel), and q = A p_new is recomputed in the update phase
// from the stored p_new instead of being kept, so the kernel holds no per-cell
// registers and runs at any size. Inter-CTA ordering uses a sense-counting grid
// barrier whose waits are bounded: a wait that gives up sets
// CFD2D_S_BARRIER_TIMEOUT and the kernel returns without further barriers.
namespace {

// The workspace solver streams its vectors through L2/HBM: 512 threads per CTA and
// two CTAs per SM (at most 64 registers a thread) keep 32 warps of loads in flight
// per SM (84 -> 54 us per iteration at 2048 x 1024 against 256 x 2 at 108 registers).
constexpr int kGridThreads = 512;
constexpr int kGridMinBlocks = 2;
constexpr int kGridUnroll = 2;  // cells a thread of the workspace solver has in flight
constexpr int kClusterL2Threads = 512;  // one 16-CTA cluster, vectors in global memory

struct GridWork {
    double* R;
    double* P0;
    double* P1;
    double* partA;
    double* partB;
    double* partC;
    unsigned int* bar;  // [0] arrival count, [1] generation
};

__device__ __forceinline__ GridWork grid_work(double* w, int n, int G) {
    GridWork W;
    W.R = w;
    W.P0 = w + n;
    W.P1 = w + 2 * (size_t)n;
    W.partA = w + 3 * (size_t)n;
    W.partB = W.partA + (size_t)G * kSlot;
    W.partC = W.partB + (size_t)G * kSlot;
    W.bar = reinterpret_cast<unsigned int*>(W.partC + (size_t)G * kSlot);
    return W;
}

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded grid barrier with one atomic per CTA (a sense-reversing counter): thread 0
// of each CTA adds 1 to the 32-bit counter, except CTA 0, which adds 2^31 - (G - 1);
// the G additions of one barrier total exactly 2^31, so the counter's top bit flips
// once, at the last arrival, and never before. Each CTA remembers the top bit it saw
// when it arrived and polls the one word until the bit differs. The counter starts
// at zero (cleared before every launch) and returns to a multiple of 2^31 after
// every barrier. A wait that gives up after about a second sets
// CFD2D_S_BARRIER_TIMEOUT and returns false (uniform over the CTA). `nblocks` is the
// number of CTAs that take part (gridDim.x, except in the self-test).
__device__ bool grid_barrier(unsigned int* bar, int* status, unsigned int nblocks) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned int add = (blockIdx.x == 0) ? (0x80000000u - (nblocks - 1u)) : 1u;
        __threadfence();
        const unsigned int seen = atomicAdd(bar, add);
        long long spins = 0;
        while (((seen ^ ld_acquire_gpu(bar)) & 0x80000000u) == 0u) {
            if (++spins > (1LL << 24)) {
                if (status) atomicOr(status, CFD2D_S_BARRIER_TIMEOUT);
                ok = 0;
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Grid-wide sum of K values: block tree, thread 0 stores the CTA partial in set
// (parity & 1) of the partial arrays (two sets, so a CTA that runs ahead into the
// next reduction never overwrites partials another CTA is still reading: it reaches
// this set again only after the barrier of the reduction in between), barrier, then
// thread t of every CTA loads partials t, t + blockDim, ... in parallel and the
// values are added by warp butterflies and a butterfly over the warp sums: one fixed
// order, so every CTA gets the same bits. Global stores a CTA made before the call
// are visible to every CTA after it (read them with __ldcg: L1 is not coherent).
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double* red_smem, double* parts, unsigned int* bar,
                                         int* status, unsigned int parity) {
    static_assert(K <= kSlot, "partial slot capacity");
    __shared__ double gsum[kSlot];
    const int G = gridDim.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    block_sum<K>(v, red_smem);
    double* set = parts + (size_t)(parity & 1u) * G * kSlot;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) set[(size_t)blockIdx.x * kSlot + k] = v[k];
    }
    if (!grid_barrier(bar, status, (unsigned int)G)) return false;
    double x[K];
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = 0.0;
    for (int b = tid; b < G; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) x[k] += __ldcg(set + (size_t)b * kSlot + k);
    }
    // every lane of a warp ends with the same bits (each butterfly stage adds the
    // same two values in both partner lanes)
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x[k] += __shfl_xor_sync(0xffffffffu, x[k], o);
    }
    const int nwg = min((int)(blockDim.x >> 5), (G + 31) >> 5);  // warps that loaded partials
    if (lane == 0 && w < nwg) {
#pragma unroll
        for (int k = 0; k < K; ++k) red_smem[k * 32 + w] = x[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double y = lane < nwg ? red_smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
            if (lane == 0) gsum[k] = y;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = gsum[k];
    // gsum and red_smem are rewritten by the next call only after its block_sum barrier
    return true;
}

// Off-diagonal entries of row (i, j): -dx2 and -dy2, or var_coef's
template <bool VAR>
struct Coef {
    double w, s, n, e;
    __device__ __forceinline__ Coef(const cfd2d_poisson& op, int i, int j) {
        if constexpr (VAR) {
            var_coef(op, i, j, w, e, s, n);
        } else {
            w = e = -op.dx2;
            s = n = -op.dy2;
        }
    }
};

// A x at cell (i, j) from a global vector (csc_matvec order)
template <bool VAR = false>
__device__ __forceinline__ double apply_A(const cfd2d_poisson& op, const double* X, int i, int j,
                                          uint8_t nb, double dg) {
    const int nx = op.nx, ny = op.ny;
    const int c = i * ny + j;
    const Coef<VAR> k(op, i, j);
    double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
    if (nb & 2) tS = k.s * X[c - 1];
    if (nb & 4) tN = k.n * X[c + 1];
    if (nb & 1) tW = k.w * X[((i == 0) ? nx - 1 : i - 1) * ny + j];
    if (nb & 8) tE = k.e * X[((i == nx - 1) ? 0 : i + 1) * ny + j];
    return row_sum(op.periodic != 0, i, nx, tW, tS, dg * X[c], tN, tE);
}

// The x neighbours of cell c = i ny + j (n = nx ny cells) found without dividing by
// ny: the periodic wrap is needed only in the first and the last row (the coupling
// bits say whether a neighbour exists at all); row is what row_sum needs of i (0,
// nx - 1, or 1 for any row in between).
struct RowPos {
    int w, e, row;
};
__device__ __forceinline__ RowPos row_pos(int c, int n, int ny, int nx) {
    const bool first = c < ny, last = c >= n - ny;
    RowPos p;
    p.w = first ? c + (n - ny) : c - ny;
    p.e = last ? c - (n - ny) : c + ny;
    p.row = first ? 0 : (last ? nx - 1 : 1);
    return p;
}

// apply_A at cell c with its RowPos (the variable coefficients still need (i, j))
template <bool VAR>
__device__ __forceinline__ double apply_A_at(const cfd2d_poisson& op, const double* X, int c, const RowPos& rp,
                                             uint8_t nb, double dg) {
    double kS = -op.dy2, kN = -op.dy2, kW = -op.dx2, kE = -op.dx2;
    if constexpr (VAR) {
        const Coef<true> k(op, c / op.ny, c % op.ny);
        kS = k.s; kN = k.n; kW = k.w; kE = k.e;
    }
    double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
    if (nb & 2) tS = kS * X[c - 1];
    if (nb & 4) tN = kN * X[c + 1];
    if (nb & 1) tW = kW * X[rp.w];
    if (nb & 8) tE = kE * X[rp.e];
    return row_sum(op.periodic != 0, rp.row, op.nx, tW, tS, dg * X[c], tN, tE);
}

}  // namespace

// Sum of K values over one thread-block cluster (any K <= kSlot, any block size that
// is a multiple of 32), pull form: warp sums, block partial stored in this CTA's own
// slot, cluster barrier, warp 0 loads the C partials through DSMEM (one per lane) and
// adds them by a butterfly, the CTA reads the sum from shared memory. Consecutive
// calls alternate two slot buffers (a slot is rewritten only after the next barrier).
template <int K>
__device__ __forceinline__ void cluster_sum_any(double (&v)[K], double* red_smem, double* slot) {
    static_assert(K <= kSlot, "slot capacity");
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __shared__ double res[kSlot];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) red_smem[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = (lane < nw) ? red_smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) slot[k] = x;
        }
    }
    cluster.sync();
    if (w == 0) {
        const double* src = cluster.map_shared_rank(slot, lane < C ? lane : 0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double y = (lane < C) ? src[k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
            if (lane == 0) res[k] = y;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = res[k];
}

// The reduction of the grid-persistent solver: over the whole cooperative grid (CL =
// false, counting barrier, may give up) or over one cluster (CL = true).
template <bool CL, int K>
__device__ __forceinline__ bool sync_sum(double (&v)[K], double* red_smem, double* parts, unsigned int* bar,
                                         int* status, double* slotA, double* slotB, int& nred) {
    if constexpr (CL) {
        cluster_sum_any<K>(v, red_smem, (nred++ & 1) ? slotB : slotA);
        return true;
    } else {
        return grid_sum<K>(v, red_smem, parts, bar, status, (unsigned int)(nred++));
    }
}

template <bool CL, bool VAR>
__global__ void __launch_bounds__(CL ? kClusterL2Threads : kGridThreads, CL ? 1 : kGridMinBlocks) k_pcg_grid(PcgLaunch L) {
    constexpr int TPB = CL ? kClusterL2Threads : kGridThreads;
    if (L.active && *L.active == 0) return;
    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const int n = nx * ny;
    const int G = gridDim.x;
    const int chunk = (n + G - 1) / G;
    const int c0 = blockIdx.x * chunk;
    const int c1 = min(n, c0 + chunk);
    GridWork W = grid_work(op.work, n, G);
    double* X = op.x0;
    double* R = W.R;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    __shared__ double red_smem[32 * kSlot];
    __shared__ double slotA[kSlot], slotB[kSlot];  // cluster mode: this CTA's partials
    int nred = 0;
    int* status = L.status_out;
#define SSUM(K, v, part) sync_sum<CL, K>(v, red_smem, part, W.bar, status, slotA, slotB, nred)

    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double csum[CFD2D_MAX_COMPONENTS + 1];
#pragma unroll
    for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) csum[k] = 0.0;
    for (int c = c0 + tid; c < c1; c += TPB) {
        const uint8_t nb = op.nbr[c];
        double braw = 0.0;
        if (nb & 0x80) {
            const int i = c / ny, j = c % ny;
            if (L.rhs_mode == 0) {
                braw = L.rhs[c];
            } else {
                const int pu = ny + 2, pv = ny + 1;
                const int ig = i + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            const int lab = op.label[c];
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) csum[k] += braw;
            if (X[c] != 0.0) csum[CFD2D_MAX_COMPONENTS] += 1.0;
        }
        R[c] = braw;
    }
    if (!SSUM(CFD2D_MAX_COMPONENTS + 1, csum, W.partA)) return;
    const bool x_any = csum[CFD2D_MAX_COMPONENTS] > 0.0;
    double part[3] = {0.0, 0.0, 0.0};
    for (int c = c0 + tid; c < c1; c += TPB) {
        const uint8_t nb = op.nbr[c];
        if (!(nb & 0x80)) { W.P1[c] = 0.0; W.P0[c] = 0.0; R[c] = 0.0; continue; }
        const int i = c / ny, j = c % ny;
        double b = R[c];
        const int lab = op.label[c];
        if (lab >= 0) {
            double mean = 0.0;
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) mean = csum[k] / op.comp_count[k];
            b = b - mean;
        }
        b = -b;
        W.P1[c] = b;
        double r = b;
        if (x_any) r = b - apply_A<VAR>(op, X, i, j, nb, op.diag[c]);
        R[c] = r;
        W.P0[c] = 0.0;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * (op.dinv[c] * r);
    }
    if (!SSUM(3, part, W.partA)) return;
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;
    if (bnrm2 == 0.0) {
        for (int c = c0 + tid; c < c1; c += TPB) X[c] = W.P1[c];
        converged = true;
    } else {
        double beta = 0.0;
        int cur = 0;
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            double* Pn = cur ? W.P1 : W.P0;
            const double* Po = cur ? W.P0 : W.P1;
            const bool first = (it == 0);
            double pq = 0.0;
            {
                // the vectors never alias: the loads of the next cells may pass this
                // cell's store (several cells' loads in flight per thread)
                const double* __restrict__ po = Po;
                double* __restrict__ pn = Pn;
                const double* __restrict__ rv = R;
                const double* __restrict__ dv = op.dinv;
                const double* __restrict__ dg = op.diag;
                const uint8_t* __restrict__ nbr = op.nbr;
#pragma unroll(kGridUnroll)
                for (int c = c0 + tid; c < c1; c += TPB) {
                    const uint8_t nb = nbr[c];
                    if (nb & 0x80) {
                        const RowPos rp = row_pos(c, n, ny, nx);
#define PNEWG(idx) (first ? (dv[idx] * rv[idx]) : (po[idx] * beta + dv[idx] * rv[idx]))
                        const double pC = PNEWG(c);
                        double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
                        double kS = mdy2, kN = mdy2, kW = mdx2, kE = mdx2;
                        if constexpr (VAR) {
                            const Coef<true> k(op, c / ny, c % ny);
                            kS = k.s; kN = k.n; kW = k.w; kE = k.e;
                        }
                        if (nb & 2) tS = kS * PNEWG(c - 1);
                        if (nb & 4) tN = kN * PNEWG(c + 1);
                        if (nb & 1) tW = kW * PNEWG(rp.w);
                        if (nb & 8) tE = kE * PNEWG(rp.e);
#undef PNEWG
                        const double qq = row_sum(op.periodic != 0, rp.row, nx, tW, tS, dg[c] * pC, tN, tE);
                        pn[c] = pC;
                        pq += pC * qq;
                    }
                }
            }
            {
                double v[1] = {pq};
                if (!SSUM(1, v, W.partA)) return;
                pq = v[0];
            }
            const double alpha = rho / pq;
            double v2[2] = {0.0, 0.0};
            {
                const double* __restrict__ pn = Pn;
                double* __restrict__ xv = X;
                double* __restrict__ rv = R;
                const double* __restrict__ dv = op.dinv;
                const double* __restrict__ dg = op.diag;
                const uint8_t* __restrict__ nbr = op.nbr;
#pragma unroll(kGridUnroll)
                for (int c = c0 + tid; c < c1; c += TPB) {
                    const uint8_t nb = nbr[c];
                    if (nb & 0x80) {
                        const double qq = apply_A_at<VAR>(op, pn, c, row_pos(c, n, ny, nx), nb, dg[c]);
                        xv[c] = xv[c] + alpha * pn[c];
                        const double r = rv[c] - alpha * qq;
                        rv[c] = r;
                        v2[0] += r * r;
                        v2[1] += r * (dv[c] * r);
                    }
                }
            }
            if (L.snap) {
                const int k = (it + 1) / L.snap_every;
                if ((it + 1) % L.snap_every == 0 && k <= L.snap_max)
                    for (int c = c0 + tid; c < c1; c += TPB) L.snap[(size_t)(k - 1) * n + c] = X[c];
            }
            if (!SSUM(2, v2, W.partA)) return;
            rr = v2[0];
            beta = v2[1] / rho;
            rho = v2[1];
            cur ^= 1;
        }
    }
    double xs[CFD2D_MAX_COMPONENTS];
#pragma unroll
    for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k) xs[k] = 0.0;
    if (op.ncomp > 0) {
        for (int c = c0 + tid; c < c1; c += TPB) {
            if (!(op.nbr[c] & 0x80)) continue;
            const int lab = op.label[c];
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) xs[k] += X[c];
        }
        if (!SSUM(CFD2D_MAX_COMPONENTS, xs, W.partA)) return;
    }
    const int pp = ny + 2;
    for (int c = c0 + tid; c < c1; c += TPB) {
        const int i = c / ny, j = c % ny;
        double pv = 0.0;
        if (op.nbr[c] & 0x80) {
            pv = X[c];
            const int lab = op.label[c];
            if (lab >= 0) {
                double mean = 0.0;
#pragma unroll
                for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                    if (k == lab) mean = xs[k] / op.comp_count[k];
                pv = pv - mean;
            }
        }
        if (!L.p_padded) {
            L.p_out[c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            if (op.periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (op.periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
            if (j == 0) L.p_out[(i + 1) * pp] = 0.0;
            if (j == ny - 1) L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
    }
    if (L.p_padded && blockIdx.x == 0) {
        for (int j = tid; j < pp; j += TPB) {
            if (!op.periodic || j == 0 || j == ny + 1) {
                L.p_out[j] = 0.0;
                L.p_out[(nx + 1) * pp + j] = 0.0;
            }
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
    if constexpr (CL) cg::this_cluster().sync();
#undef SSUM
}

// ---------------------------------------------------------------- slab solver
// The grid-persistent solver for grids beyond one cluster whose state still fits in
// the shared memory of one CTA per SM (k_pcg_slab): CTA b owns a slab of whole rows
// and keeps x, r, z, p (two buffers), 1/diag, diag and the coupling bits of its cells
// on chip for the whole solve, as the cluster solver does; only the first and last
// row of each slab cross to its two neighbours, through global memory (L2), and the
// dot products are reduced over the grid by grid_sum (one atomic per CTA). Per iteration:
// phase A (p = z + beta p, q = A p, p.q partial; the slab's boundary rows of p are
// published), reduction 1, the neighbours' boundary rows of p are read; phase B (x, r,
// z update, r.r and r.z partials; boundary rows of z published), reduction 2, the
// neighbours' boundary rows of z are read. Same iteration form and operation order as
// the other forms (scipy's, csc_matvec row order).
namespace {

constexpr int kSlabThreads = 512;
constexpr int kHaloRegs = 4;  // halo values per thread: two rows of ny <= 2 * kSlabThreads

}  // namespace

// Shared memory of one slab: seven doubles and one byte per own cell, two halo rows
// of z and two of p (the latter hold x0 in the prologue).
size_t pcg_slab_smem_bytes(int cap, int ny) { return (size_t)cap * (kArrays * sizeof(double) + 1) + 4 * (size_t)ny * sizeof(double) + 16; }

template <int CPT>
__global__ void __launch_bounds__(kSlabThreads, 1) k_pcg_slab(PcgLaunch L) {
    if (L.active && *L.active == 0) return;  // uniform over the grid
    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int G = gridDim.x, me = blockIdx.x;
    const int r0 = row0_of(me, nx, G), r1 = row0_of(me + 1, nx, G);
    const int rows = r1 - r0;
    const int nloc = rows * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    const int goff = r0 * ny;
    const int n = nx * ny;

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* R = X + cap;
    double* P0 = R + cap;
    double* P1 = P0 + cap;
    double* DI = P1 + cap;
    double* DG = DI + cap;
    double* Z = DG + cap;
    double* HZ = Z + cap;        // z of the west halo row at [0, ny), of the east one at [ny, 2 ny)
    double* HP = HZ + 2 * ny;    // p of the halo rows (x0 in the prologue), same layout
    uint8_t* NB = reinterpret_cast<uint8_t*>(HP + 2 * ny);
    __shared__ double red_smem[32 * kSlot];
    __shared__ double cmean[CFD2D_MAX_COMPONENTS];
    // global exchange rows and reduction slots in the workspace
    double* GZ = op.work;
    double* GP = op.work + n;
    double* parts = op.work + 3 * (size_t)n;
    unsigned int* bar = reinterpret_cast<unsigned int*>(parts + (size_t)2 * G * kSlot);
    unsigned int seq = 0;
    int* status = L.status_out;
    const int iw = (r0 == 0) ? (periodic ? nx - 1 : -1) : r0 - 1;
    const int ie = (r1 == nx) ? (periodic ? 0 : -1) : r1;
    const unsigned magic = (unsigned)(((1ull << 32) + (unsigned)ny - 1) / (unsigned)ny);

    // ------------------------------------------------------------ prologue
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double csum[CFD2D_MAX_COMPONENTS + 1];
#pragma unroll
    for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) csum[k] = 0.0;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const int gidx = goff + c;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        const double x0 = op.x0[gidx];
        X[c] = x0;
        DI[c] = op.dinv[gidx];
        DG[c] = op.diag[gidx];
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                // div(F, G) / dt at interior cell (i+1, j+1) (cfd2d/solver.py:264-266)
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                const int pu = ny + 2, pv = ny + 1;
                const int ig = r0 + li + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            const int lab = op.ncomp > 0 ? op.label[gidx] : -1;
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) csum[k] += braw;
            if (x0 != 0.0) csum[CFD2D_MAX_COMPONENTS] += 1.0;
        }
        R[c] = braw;
    }
    // x0 of the halo rows: written by the caller before the launch, rewritten by this
    // kernel only in its epilogue, which no CTA reaches before every CTA is past here
    for (int t = tid; t < 2 * ny; t += kSlabThreads) {
        const int row = t < ny ? iw : ie;
        HP[t] = row >= 0 ? op.x0[(size_t)row * ny + (t < ny ? t : t - ny)] : 0.0;
    }
    // scipy computes A x0 only if x0 has a nonzero; Neumann-component sums of b
    if (!grid_sum<CFD2D_MAX_COMPONENTS + 1>(csum, red_smem, parts, bar, status, ++seq)) return;
    const bool x_any = csum[CFD2D_MAX_COMPONENTS] > 0.0;
    const int ncomp = op.ncomp;
    if (tid < ncomp) cmean[tid] = csum[tid] / op.comp_count[tid];
    __syncthreads();

    double part[3] = {0.0, 0.0, 0.0};
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const uint8_t nb = NB[c];
        if (!(nb & 0x80)) { P1[c] = 0.0; P0[c] = 0.0; R[c] = 0.0; Z[c] = 0.0; continue; }
        double b = R[c];
        if (ncomp > 0) {
            const int lab = op.label[goff + c];
            if (lab >= 0) b = b - cmean[lab];
        }
        b = -b;
        P1[c] = b;  // kept for the ||b|| == 0 return
        double r = b;
        if (x_any) {
            const int li = (int)__umulhi((unsigned)c, magic);
            const int j = c - li * ny;
            double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
            if (nb & 2) tS = mdy2 * X[c - 1];
            if (nb & 4) tN = mdy2 * X[c + 1];
            if (nb & 1) tW = mdx2 * ((li > 0) ? X[c - ny] : HP[j]);
            if (nb & 8) tE = mdx2 * ((li < rows - 1) ? X[c + ny] : HP[ny + j]);
            r = b - row_sum(periodic, r0 + li, nx, tW, tS, DG[c] * X[c], tN, tE);
        }
        R[c] = r;
        P0[c] = 0.0;
        const double z = DI[c] * r;
        Z[c] = z;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * z;
    }
    __syncthreads();
    // boundary rows of z for the neighbours (iteration 0 reads z of the halo rows)
    for (int t = tid; t < 2 * ny; t += kSlabThreads) {
        const int lr = t < ny ? 0 : rows - 1;
        const int j = t < ny ? t : t - ny;
        GZ[(size_t)(r0 + lr) * ny + j] = Z[lr * ny + j];
    }
    if (!grid_sum<3>(part, red_smem, parts, bar, status, ++seq)) return;
    // halo rows of z and p go through registers: the loads are issued right after a
    // reduction and stored to shared memory only where they are needed, so their
    // latency overlaps the cells that do not need them
    double hz[kHaloRegs], hp[kHaloRegs];
    auto load_halo = [&](double (&h)[kHaloRegs], const double* src) {
#pragma unroll
        for (int u = 0; u < kHaloRegs; ++u) {
            const int t = tid + u * kSlabThreads;
            const int row = t < ny ? iw : ie;
            h[u] = (t < 2 * ny && row >= 0) ? __ldcg(src + (size_t)row * ny + (t < ny ? t : t - ny)) : 0.0;
        }
    };
    auto store_halo = [&](const double (&h)[kHaloRegs], double* dst) {
#pragma unroll
        for (int u = 0; u < kHaloRegs; ++u) {
            const int t = tid + u * kSlabThreads;
            if (t < 2 * ny) dst[t] = h[u];
        }
    };
    load_halo(hz, GZ);
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;
    if (bnrm2 == 0.0) {
        for (int c = tid; c < nloc; c += kSlabThreads) X[c] = P1[c];
        converged = true;
    } else {
        double beta = 0.0;
        int cur = 0;
        double q[2 * CPT];
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            double* Pn = cur ? P1 : P0;
            const double* Po = cur ? P0 : P1;
            const bool first = (it == 0);
            double pq = 0.0;
            // two cells (c, c+1) of one row per slot; ny is even, so c is even and
            // every 16-byte pair load is aligned. Pass 0 takes the pairs of the slab's
            // inner rows, pass 1 (after the halo z reaches shared memory) the pairs of
            // its first and last rows.
            auto pair_a = [&](int k, int pass) {
                const int c = 2 * (tid + k * kSlabThreads);
                if (c >= nloc) return;
                const int li = (int)__umulhi((unsigned)c, magic);
                const bool edge = (li == 0) || (li == rows - 1);
                if (edge != (pass == 1)) return;
                q[2 * k] = 0.0;
                q[2 * k + 1] = 0.0;
                const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                const unsigned nb0 = nb2 & 0xFFu, nb1 = nb2 >> 8;
                if (!((nb0 | nb1) & 0x80u)) return;
                const int j = c - li * ny;
                const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                double pC0 = z2.x, pC1 = z2.y;
                if (!first) {
                    const double2 o2 = *reinterpret_cast<const double2*>(Po + c);
                    pC0 = o2.x * beta + z2.x;
                    pC1 = o2.y * beta + z2.y;
                }
                // solid cells carry p = z = 0 and no coupling bits, so their terms vanish
                double tW0 = 0.0, tW1 = 0.0, tE0 = 0.0, tE1 = 0.0;
                const double tS0 = (nb0 & 2) ? mdy2 * (first ? Z[c - 1] : Po[c - 1] * beta + Z[c - 1]) : 0.0;
                const double tN0 = (nb0 & 4) ? mdy2 * pC1 : 0.0;
                const double tS1 = (nb1 & 2) ? mdy2 * pC0 : 0.0;
                const double tN1 = (nb1 & 4) ? mdy2 * (first ? Z[c + 2] : Po[c + 2] * beta + Z[c + 2]) : 0.0;
                if ((nb0 | nb1) & 1) {
                    const bool own = li > 0;
                    const double2 gz = *reinterpret_cast<const double2*>(own ? (Z + c - ny) : (HZ + j));
                    double w0 = gz.x, w1 = gz.y;
                    if (!first) {
                        const double2 go = *reinterpret_cast<const double2*>(own ? (Po + c - ny) : (HP + j));
                        w0 = go.x * beta + gz.x;
                        w1 = go.y * beta + gz.y;
                    }
                    if (nb0 & 1) tW0 = mdx2 * w0;
                    if (nb1 & 1) tW1 = mdx2 * w1;
                }
                if ((nb0 | nb1) & 8) {
                    const bool own = li < rows - 1;
                    const double2 gz = *reinterpret_cast<const double2*>(own ? (Z + c + ny) : (HZ + ny + j));
                    double e0 = gz.x, e1 = gz.y;
                    if (!first) {
                        const double2 go = *reinterpret_cast<const double2*>(own ? (Po + c + ny) : (HP + ny + j));
                        e0 = go.x * beta + gz.x;
                        e1 = go.y * beta + gz.y;
                    }
                    if (nb0 & 8) tE0 = mdx2 * e0;
                    if (nb1 & 8) tE1 = mdx2 * e1;
                }
                const double2 dg = *reinterpret_cast<const double2*>(DG + c);
                const int i = r0 + li;
                const double q0 = row_sum(periodic, i, nx, tW0, tS0, dg.x * pC0, tN0, tE0);
                const double q1 = row_sum(periodic, i, nx, tW1, tS1, dg.y * pC1, tN1, tE1);
                *reinterpret_cast<double2*>(Pn + c) = make_double2(pC0, pC1);
                q[2 * k] = q0;
                q[2 * k + 1] = q1;
                pq += pC0 * q0;
                pq += pC1 * q1;
            };
#pragma unroll
            for (int k = 0; k < CPT; ++k) pair_a(k, 0);
            store_halo(hz, HZ);
            __syncthreads();
#pragma unroll
            for (int k = 0; k < CPT; ++k) pair_a(k, 1);
            __syncthreads();
            // boundary rows of the new p: the neighbours' p_old of the next iteration
            for (int t = tid; t < 2 * ny; t += kSlabThreads) {
                const int lr = t < ny ? 0 : rows - 1;
                const int j = t < ny ? t : t - ny;
                GP[(size_t)(r0 + lr) * ny + j] = Pn[lr * ny + j];
            }
            {
                double v[1] = {pq};
                if (!grid_sum<1>(v, red_smem, parts, bar, status, ++seq)) return;
                pq = v[0];
            }
            // the halo rows' new p: phase B does not read HP, the next phase A does
            load_halo(hp, GP);
            const double alpha = rho / pq;
            double v2[2] = {0.0, 0.0};
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = 2 * (tid + k * kSlabThreads);
                if (c >= nloc) continue;
                const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                const bool f0 = nb2 & 0x80u, f1 = (nb2 >> 8) & 0x80u;
                if (!(f0 || f1)) continue;
                double2 x2 = *reinterpret_cast<const double2*>(X + c);
                double2 r2 = *reinterpret_cast<const double2*>(R + c);
                double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                const double2 p2 = *reinterpret_cast<const double2*>(Pn + c);
                const double2 d2 = *reinterpret_cast<const double2*>(DI + c);
                if (f0) {
                    x2.x = x2.x + alpha * p2.x;
                    r2.x = r2.x - alpha * q[2 * k];
                    z2.x = d2.x * r2.x;
                    v2[0] += r2.x * r2.x;
                    v2[1] += r2.x * z2.x;
                }
                if (f1) {
                    x2.y = x2.y + alpha * p2.y;
                    r2.y = r2.y - alpha * q[2 * k + 1];
                    z2.y = d2.y * r2.y;
                    v2[0] += r2.y * r2.y;
                    v2[1] += r2.y * z2.y;
                }
                *reinterpret_cast<double2*>(X + c) = x2;
                *reinterpret_cast<double2*>(R + c) = r2;
                *reinterpret_cast<double2*>(Z + c) = z2;
            }
            // phase A of this iteration is done with HP (the barrier of the p.q
            // reduction); the next one reads it after the barriers below
            store_halo(hp, HP);
            __syncthreads();
            for (int t = tid; t < 2 * ny; t += kSlabThreads) {
                const int lr = t < ny ? 0 : rows - 1;
                const int j = t < ny ? t : t - ny;
                GZ[(size_t)(r0 + lr) * ny + j] = Z[lr * ny + j];
            }
            if (!grid_sum<2>(v2, red_smem, parts, bar, status, ++seq)) return;
            // phase A of this iteration is done with HZ; the next stores the new rows
            load_halo(hz, GZ);
            rr = v2[0];
            beta = v2[1] / rho;
            rho = v2[1];
            cur ^= 1;
        }
    }
    // ------------------------------------------------------------ epilogue
    __syncthreads();
    double xs[CFD2D_MAX_COMPONENTS];
#pragma unroll
    for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k) xs[k] = 0.0;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        op.x0[goff + c] = X[c];
        if (op.ncomp > 0 && (NB[c] & 0x80)) {
            const int lab = op.label[goff + c];
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) xs[k] += X[c];
        }
    }
    if (ncomp > 0) {
        if (!grid_sum<CFD2D_MAX_COMPONENTS>(xs, red_smem, parts, bar, status, ++seq)) return;
        if (tid < ncomp) cmean[tid] = xs[tid] / op.comp_count[tid];
    }
    __syncthreads();
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const int li = (int)__umulhi((unsigned)c, magic);
        const int j = c - li * ny;
        const int i = r0 + li;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) pv = pv - cmean[lab];
            }
        }
        if (!L.p_padded) {
            L.p_out[goff + c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            // periodic ghost rows: p[0,:] = p[nx,:], p[nx+1,:] = p[1,:]
            if (periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
        }
    }
    if (L.p_padded) {
        for (int i = r0 + tid; i < r1; i += kSlabThreads) {
            L.p_out[(i + 1) * pp] = 0.0;
            L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
        if (me == 0) {
            for (int j = tid; j < pp; j += kSlabThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
        }
        if (me == G - 1) {
            for (int j = tid; j < pp; j += kSlabThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
}

// Single-reduction form of the slab solver (k_pcg_slab1): the same layout, with the
// Jacobi-PCG recurrence of Chronopoulos and Gear (1989), which needs one grid-wide
// reduction per iteration instead of two. Each iteration updates p = z + beta p,
// q = w + beta q (= A p), x, r and z = D^-1 r of the slab's own cells, publishes the
// slab's boundary rows of z with a per-CTA sequence word (release store), computes
// w = A z on the inner rows while those rows travel, waits (bounded) for the two
// neighbours' words, finishes w on its first and last row and reduces r.z, z.w and
// r.r together; p.q = z.w - beta r.z / alpha_prev. In exact arithmetic the iterates
// are scipy's; in floating point they round differently (measured on the CPU with
// the oracle: the 2000-step 64 x 64 cavity stays within 1e-11 of the reference with
// CG iteration counts within 2; on the device at 1024 x 512 the same iteration
// counts as scipy, u and v within 1e-12, p within 2.4e-9 after the first step).
// Selected by grid_ctas = -2; the default slab form keeps scipy's two reductions.
template <int CPT>
__global__ void __launch_bounds__(kSlabThreads, 1) k_pcg_slab1(PcgLaunch L) {
    if (L.active && *L.active == 0) return;  // uniform over the grid
    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int G = gridDim.x, me = blockIdx.x;
    const int r0 = row0_of(me, nx, G), r1 = row0_of(me + 1, nx, G);
    const int rows = r1 - r0;
    const int nloc = rows * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;
    const int goff = r0 * ny;
    const int n = nx * ny;

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* R = X + cap;
    double* P0 = R + cap;   // p (P1 holds b until the first iteration)
    double* P1 = P0 + cap;  // q = A p, by its recurrence
    double* DI = P1 + cap;
    double* DG = DI + cap;
    double* Z = DG + cap;
    double* HZ = Z + cap;        // z of the west halo row at [0, ny), of the east one at [ny, 2 ny)
    double* HP = HZ + 2 * ny;    // x0 of the halo rows (prologue only), same layout
    uint8_t* NB = reinterpret_cast<uint8_t*>(HP + 2 * ny);
    __shared__ double red_smem[32 * kSlot];
    __shared__ double cmean[CFD2D_MAX_COMPONENTS];
    // global exchange rows and reduction slots in the workspace
    double* GZ = op.work;
    // one sequence word per CTA (boundary rows of z published), after the barrier word
    double* parts = op.work + 3 * (size_t)n;
    unsigned int* bar = reinterpret_cast<unsigned int*>(parts + (size_t)2 * G * kSlot);
    unsigned int* zflag = bar + 2;
    unsigned int seq = 0;
    int* status = L.status_out;
    const int iw = (r0 == 0) ? (periodic ? nx - 1 : -1) : r0 - 1;
    const int ie = (r1 == nx) ? (periodic ? 0 : -1) : r1;
    const unsigned magic = (unsigned)(((1ull << 32) + (unsigned)ny - 1) / (unsigned)ny);

    // ------------------------------------------------------------ prologue
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double csum[CFD2D_MAX_COMPONENTS + 1];
#pragma unroll
    for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) csum[k] = 0.0;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const int gidx = goff + c;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        const double x0 = op.x0[gidx];
        X[c] = x0;
        DI[c] = op.dinv[gidx];
        DG[c] = op.diag[gidx];
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                // div(F, G) / dt at interior cell (i+1, j+1) (cfd2d/solver.py:264-266)
                const int li = (int)__umulhi((unsigned)c, magic);
                const int j = c - li * ny;
                const int pu = ny + 2, pv = ny + 1;
                const int ig = r0 + li + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            const int lab = op.ncomp > 0 ? op.label[gidx] : -1;
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) csum[k] += braw;
            if (x0 != 0.0) csum[CFD2D_MAX_COMPONENTS] += 1.0;
        }
        R[c] = braw;
    }
    // x0 of the halo rows: written by the caller before the launch, rewritten by this
    // kernel only in its epilogue, which no CTA reaches before every CTA is past here
    for (int t = tid; t < 2 * ny; t += kSlabThreads) {
        const int row = t < ny ? iw : ie;
        HP[t] = row >= 0 ? op.x0[(size_t)row * ny + (t < ny ? t : t - ny)] : 0.0;
    }
    // scipy computes A x0 only if x0 has a nonzero; Neumann-component sums of b
    if (!grid_sum<CFD2D_MAX_COMPONENTS + 1>(csum, red_smem, parts, bar, status, ++seq)) return;
    const bool x_any = csum[CFD2D_MAX_COMPONENTS] > 0.0;
    const int ncomp = op.ncomp;
    if (tid < ncomp) cmean[tid] = csum[tid] / op.comp_count[tid];
    __syncthreads();

    double part[3] = {0.0, 0.0, 0.0};
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const uint8_t nb = NB[c];
        if (!(nb & 0x80)) { P1[c] = 0.0; P0[c] = 0.0; R[c] = 0.0; Z[c] = 0.0; continue; }
        double b = R[c];
        if (ncomp > 0) {
            const int lab = op.label[goff + c];
            if (lab >= 0) b = b - cmean[lab];
        }
        b = -b;
        P1[c] = b;  // kept for the ||b|| == 0 return
        double r = b;
        if (x_any) {
            const int li = (int)__umulhi((unsigned)c, magic);
            const int j = c - li * ny;
            double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
            if (nb & 2) tS = mdy2 * X[c - 1];
            if (nb & 4) tN = mdy2 * X[c + 1];
            if (nb & 1) tW = mdx2 * ((li > 0) ? X[c - ny] : HP[j]);
            if (nb & 8) tE = mdx2 * ((li < rows - 1) ? X[c + ny] : HP[ny + j]);
            r = b - row_sum(periodic, r0 + li, nx, tW, tS, DG[c] * X[c], tN, tE);
        }
        R[c] = r;
        P0[c] = 0.0;
        const double z = DI[c] * r;
        Z[c] = z;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * z;
    }
    __syncthreads();
    __syncthreads();
    // boundary rows of z for the neighbours, then the grid reduction of b.b, r.r, r.z
    for (int t = tid; t < 2 * ny; t += kSlabThreads) {
        const int lr = t < ny ? 0 : rows - 1;
        const int j = t < ny ? t : t - ny;
        GZ[(size_t)(r0 + lr) * ny + j] = Z[lr * ny + j];
    }
    if (!grid_sum<3>(part, red_smem, parts, bar, status, ++seq)) return;
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;
    // w = A z of the thread's cell pairs, kept in registers until the next update
    double w[2 * CPT];
    // row-sum of A z at pair c (cells c, c + 1 of local row li) from shared memory
    auto az_pair = [&](int c, int li, double& w0, double& w1) {
        const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
        const unsigned nb0 = nb2 & 0xFFu, nb1 = nb2 >> 8;
        w0 = 0.0;
        w1 = 0.0;
        if (!((nb0 | nb1) & 0x80u)) return;
        const int j = c - li * ny;
        const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
        double tW0 = 0.0, tW1 = 0.0, tE0 = 0.0, tE1 = 0.0;
        const double tS0 = (nb0 & 2) ? mdy2 * Z[c - 1] : 0.0;
        const double tN0 = (nb0 & 4) ? mdy2 * z2.y : 0.0;
        const double tS1 = (nb1 & 2) ? mdy2 * z2.x : 0.0;
        const double tN1 = (nb1 & 4) ? mdy2 * Z[c + 2] : 0.0;
        if ((nb0 | nb1) & 1) {
            const double2 g = *reinterpret_cast<const double2*>(li > 0 ? (Z + c - ny) : (HZ + j));
            if (nb0 & 1) tW0 = mdx2 * g.x;
            if (nb1 & 1) tW1 = mdx2 * g.y;
        }
        if ((nb0 | nb1) & 8) {
            const double2 g = *reinterpret_cast<const double2*>(li < rows - 1 ? (Z + c + ny) : (HZ + ny + j));
            if (nb0 & 8) tE0 = mdx2 * g.x;
            if (nb1 & 8) tE1 = mdx2 * g.y;
        }
        const double2 dg = *reinterpret_cast<const double2*>(DG + c);
        const int i = r0 + li;
        w0 = row_sum(periodic, i, nx, tW0, tS0, dg.x * z2.x, tN0, tE0);
        w1 = row_sum(periodic, i, nx, tW1, tS1, dg.y * z2.y, tN1, tE1);
    };
    // neighbours' boundary rows of z for sequence number zs: wait (bounded) for their
    // words, then load the rows into HZ. Returns false on a timeout (uniform).
    auto halo_z = [&](unsigned int zs) -> bool {
        __shared__ int hok;
        if (tid < 2) {
            const int row = tid == 0 ? iw : ie;
            int okl = 1;
            if (row >= 0) {
                const int o = owner_of(row, nx, G);
                long long spins = 0;
                while ((int)(ld_acquire_gpu(zflag + o) - zs) < 0) {
                    if (++spins > (1LL << 24)) {
                        okl = 0;
                        if (status) atomicOr(status, CFD2D_S_BARRIER_TIMEOUT);
                        break;
                    }
                }
                __threadfence();
            }
            if (tid == 0) hok = 1;
            __syncwarp(0x3u);
            if (!okl) hok = 0;
        }
        __syncthreads();
        if (!hok) return false;
        for (int t = tid; t < 2 * ny; t += kSlabThreads) {
            const int row = t < ny ? iw : ie;
            HZ[t] = row >= 0 ? __ldcg(GZ + (size_t)row * ny + (t < ny ? t : t - ny)) : 0.0;
        }
        __syncthreads();
        return true;
    };
    // w and delta = z.w of the initial z (the grid reduction above made every CTA's
    // boundary rows of z visible; sequence 0 needs no wait)
    double delta;
    {
        for (int t = tid; t < 2 * ny; t += kSlabThreads) {
            const int row = t < ny ? iw : ie;
            HZ[t] = row >= 0 ? __ldcg(GZ + (size_t)row * ny + (t < ny ? t : t - ny)) : 0.0;
        }
        __syncthreads();
        double d[1] = {0.0};
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int c = 2 * (tid + k * kSlabThreads);
            if (c >= nloc) { w[2 * k] = w[2 * k + 1] = 0.0; continue; }
            const int li = (int)__umulhi((unsigned)c, magic);
            az_pair(c, li, w[2 * k], w[2 * k + 1]);
            const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
            d[0] += z2.x * w[2 * k];
            d[0] += z2.y * w[2 * k + 1];
        }
        if (!grid_sum<1>(d, red_smem, parts, bar, status, ++seq)) return;
        delta = d[0];
    }
    if (bnrm2 == 0.0) {
        for (int c = tid; c < nloc; c += kSlabThreads) X[c] = P1[c];
        converged = true;
    } else {
        double rho_prev = 1.0, alpha_prev = 1.0;
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            const bool first = (it == 0);
            // single-reduction recurrence (Chronopoulos and Gear): p = z + beta p,
            // q = w + beta q (= A p), p.q = delta - beta rho / alpha_prev
            double beta = 0.0, pq = delta;
            if (!first) {
                beta = rho / rho_prev;
                pq = delta - (beta * rho) / alpha_prev;
            }
            const double alpha = rho / pq;
            double v3[3] = {0.0, 0.0, 0.0};  // r.z, z.w, r.r
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = 2 * (tid + k * kSlabThreads);
                if (c >= nloc) continue;
                const unsigned nb2 = *reinterpret_cast<const uint16_t*>(NB + c);
                const bool f0 = nb2 & 0x80u, f1 = (nb2 >> 8) & 0x80u;
                if (!(f0 || f1)) continue;
                double2 x2 = *reinterpret_cast<const double2*>(X + c);
                double2 r2 = *reinterpret_cast<const double2*>(R + c);
                double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                double2 p2 = *reinterpret_cast<const double2*>(P0 + c);
                double2 q2 = *reinterpret_cast<const double2*>(P1 + c);
                const double2 d2 = *reinterpret_cast<const double2*>(DI + c);
                if (first) {
                    p2 = z2;
                    q2 = make_double2(w[2 * k], w[2 * k + 1]);
                } else {
                    p2 = make_double2(p2.x * beta + z2.x, p2.y * beta + z2.y);
                    q2 = make_double2(q2.x * beta + w[2 * k], q2.y * beta + w[2 * k + 1]);
                }
                if (f0) {
                    x2.x = x2.x + alpha * p2.x;
                    r2.x = r2.x - alpha * q2.x;
                    z2.x = d2.x * r2.x;
                    v3[0] += r2.x * z2.x;
                    v3[2] += r2.x * r2.x;
                }
                if (f1) {
                    x2.y = x2.y + alpha * p2.y;
                    r2.y = r2.y - alpha * q2.y;
                    z2.y = d2.y * r2.y;
                    v3[0] += r2.y * z2.y;
                    v3[2] += r2.y * r2.y;
                }
                *reinterpret_cast<double2*>(X + c) = x2;
                *reinterpret_cast<double2*>(R + c) = r2;
                *reinterpret_cast<double2*>(Z + c) = z2;
                *reinterpret_cast<double2*>(P0 + c) = p2;
                *reinterpret_cast<double2*>(P1 + c) = q2;
            }
            __syncthreads();
            // boundary rows of the new z, then this CTA's sequence word (release)
            for (int t = tid; t < 2 * ny; t += kSlabThreads) {
                const int lr = t < ny ? 0 : rows - 1;
                const int j = t < ny ? t : t - ny;
                GZ[(size_t)(r0 + lr) * ny + j] = Z[lr * ny + j];
            }
            __syncthreads();
            const unsigned int zs = (unsigned int)it + 1u;
            if (tid == 0) {
                __threadfence();
                asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(zflag + me), "r"(zs) : "memory");
            }
            // w = A z of the inner rows while the neighbours' rows travel
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = 2 * (tid + k * kSlabThreads);
                if (c >= nloc) { w[2 * k] = w[2 * k + 1] = 0.0; continue; }
                const int li = (int)__umulhi((unsigned)c, magic);
                if (li == 0 || li == rows - 1) continue;
                az_pair(c, li, w[2 * k], w[2 * k + 1]);
                const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                v3[1] += z2.x * w[2 * k];
                v3[1] += z2.y * w[2 * k + 1];
            }
            if (!halo_z(zs)) return;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = 2 * (tid + k * kSlabThreads);
                if (c >= nloc) continue;
                const int li = (int)__umulhi((unsigned)c, magic);
                if (!(li == 0 || li == rows - 1)) continue;
                az_pair(c, li, w[2 * k], w[2 * k + 1]);
                const double2 z2 = *reinterpret_cast<const double2*>(Z + c);
                v3[1] += z2.x * w[2 * k];
                v3[1] += z2.y * w[2 * k + 1];
            }
            if (!grid_sum<3>(v3, red_smem, parts, bar, status, ++seq)) return;
            rho_prev = rho;
            alpha_prev = alpha;
            rho = v3[0];
            delta = v3[1];
            rr = v3[2];
        }
    }
    // ------------------------------------------------------------ epilogue
    __syncthreads();
    double xs[CFD2D_MAX_COMPONENTS];
#pragma unroll
    for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k) xs[k] = 0.0;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        op.x0[goff + c] = X[c];
        if (op.ncomp > 0 && (NB[c] & 0x80)) {
            const int lab = op.label[goff + c];
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) xs[k] += X[c];
        }
    }
    if (ncomp > 0) {
        if (!grid_sum<CFD2D_MAX_COMPONENTS>(xs, red_smem, parts, bar, status, ++seq)) return;
        if (tid < ncomp) cmean[tid] = xs[tid] / op.comp_count[tid];
    }
    __syncthreads();
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kSlabThreads) {
        const int li = (int)__umulhi((unsigned)c, magic);
        const int j = c - li * ny;
        const int i = r0 + li;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            if (ncomp > 0) {
                const int lab = op.label[goff + c];
                if (lab >= 0) pv = pv - cmean[lab];
            }
        }
        if (!L.p_padded) {
            L.p_out[goff + c] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            // periodic ghost rows: p[0,:] = p[nx,:], p[nx+1,:] = p[1,:]
            if (periodic && i == nx - 1) L.p_out[j + 1] = pv;
            if (periodic && i == 0) L.p_out[(nx + 1) * pp + j + 1] = pv;
        }
    }
    if (L.p_padded) {
        for (int i = r0 + tid; i < r1; i += kSlabThreads) {
            L.p_out[(i + 1) * pp] = 0.0;
            L.p_out[(i + 1) * pp + ny + 1] = 0.0;
        }
        if (me == 0) {
            for (int j = tid; j < pp; j += kSlabThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
        }
        if (me == G - 1) {
            for (int j = tid; j < pp; j += kSlabThreads)
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
}

namespace {

constexpr int kMaxDevices = 64;

// SM count and opt-in shared memory per block of the current device, looked up once
// per device (0 SMs: the lookup failed).
struct DevLimits {
    int sms = 0, smem_optin = 0, dev = -1;
};
DevLimits dev_limits() {
    static DevLimits cache[kMaxDevices];
    DevLimits d;
    if (cudaGetDevice(&d.dev) != cudaSuccess || d.dev < 0) return DevLimits{};
    if (d.dev < kMaxDevices && cache[d.dev].sms > 0) return cache[d.dev];
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, d.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.dev) != cudaSuccess)
        return DevLimits{};
    if (d.dev < kMaxDevices) cache[d.dev] = d;
    return d;
}

// CTAs of the workspace solver: every SM times the CTAs that fit on one, at most
// one per kGridThreads cells; per device.
template <bool VAR>
int grid_blocks_for(int n) {
    static int per_sm_cache[kMaxDevices];
    const DevLimits d = dev_limits();
    if (d.sms <= 0) return 0;
    int per_sm = d.dev < kMaxDevices ? per_sm_cache[d.dev] : 0;
    if (per_sm <= 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_grid<false, VAR>, kGridThreads, 0) !=
            cudaSuccess)
            return 0;
        if (d.dev < kMaxDevices) per_sm_cache[d.dev] = per_sm;
    }
    long long g = (long long)per_sm * d.sms;
    const long long need = (n + kGridThreads - 1) / kGridThreads;
    if (g > need) g = need;
    if (g < 1) g = 1;
    return (int)g;
}

// Cell pairs per thread of the slab solver for `cap` cells per CTA (0: too many).
int slab_cpt_for(int cap) {
    const int need = ((cap + 1) / 2 + kSlabThreads - 1) / kSlabThreads;
    if (need <= 1) return 1;
    if (need <= 2) return 2;
    if (need <= 4) return 4;
    if (need <= 8) return 8;
    return 0;
}

// The slab solver's launch for an nx x ny constant-coefficient grid: one CTA per SM
// (at most one per row) when ny is even and a slab of ceil(nx / G) rows fits in the
// opt-in shared memory beside the kernel's static arrays. False: use the workspace form.
bool slab_plan(int nx, int ny, int* G_out, int* cap_out) {
    if (ny % 2 != 0 || 2 * ny > kHaloRegs * kSlabThreads) return false;
    const DevLimits d = dev_limits();
    if (d.sms <= 0) return false;
    const int G = nx < d.sms ? nx : d.sms;
    if (G < 2) return false;
    const int cap = ((nx + G - 1) / G) * ny;
    const size_t static_bytes = (32 * kSlot + kSlot + CFD2D_MAX_COMPONENTS) * sizeof(double) + 1024;
    if (pcg_slab_smem_bytes(cap, ny) + static_bytes > (size_t)d.smem_optin) return false;
    if (slab_cpt_for(cap) == 0) return false;
    *G_out = G;
    *cap_out = cap;
    return true;
}

template <int CPT, bool SINGLE>
cudaError_t launch_slab(const PcgLaunch& L0, int G, int cap, cudaStream_t s) {
    static bool configured[kMaxDevices];
    auto kern = SINGLE ? k_pcg_slab1<CPT> : k_pcg_slab<CPT>;
    const DevLimits d = dev_limits();
    if (d.sms <= 0 || d.dev >= kMaxDevices) return cudaErrorInvalidDevice;
    const size_t bytes = pcg_slab_smem_bytes(cap, L0.op.ny);
    if (!configured[d.dev]) {
        const int dyn = d.smem_optin - (int)((32 * kSlot + kSlot + CFD2D_MAX_COMPONENTS) * sizeof(double)) - 1024;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        if (e != cudaSuccess) return e;
        configured[d.dev] = true;
    }
    PcgLaunch L = L0;
    L.cap_cells = cap;
    const size_t n = (size_t)L.op.nx * L.op.ny;
    // the barrier counter (and the single-reduction form's per-CTA sequence words)
    // start from zero on every launch, whatever an earlier launch that gave up on a
    // wait left behind
    cudaError_t e = cudaMemsetAsync(L.op.work + 3 * n + (size_t)2 * G * kSlot, 0,
                                    sizeof(double) + (size_t)G * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    void* args[] = {&L};
    return cudaLaunchCooperativeKernel((const void*)kern, dim3(G), dim3(kSlabThreads), args, bytes, s);
}

}  // namespace

// The bounded grid barrier of the persistent solvers on a grid of one block, with the
// barrier words as the caller set them (cfd2d_barrier_selftest).
__global__ void k_barrier_probe(unsigned int* bar, int* status, int* ok_out) {
    const unsigned int expected = bar[1] > 0u ? bar[1] : 1u;
    const bool ok = grid_barrier(bar, status, expected);
    if (threadIdx.x == 0) *ok_out = ok ? 1 : 0;
}

cudaError_t barrier_selftest(unsigned int* bar, int* status, int* ok_out, cudaStream_t s) {
    k_barrier_probe<<<1, 32, 0, s>>>(bar, status, ok_out);
    return cudaGetLastError();
}

__global__ void k_matvec(cfd2d_poisson op, const double* x, double* y) {
    const int n = op.nx * op.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint8_t nb = op.nbr[c];
        if (!(nb & 0x80)) { y[c] = 0.0; continue; }
        y[c] = op.bx ? apply_A<true>(op, x, c / op.ny, c % op.ny, nb, op.diag[c])
                     : apply_A<false>(op, x, c / op.ny, c % op.ny, nb, op.diag[c]);
    }
}

cudaError_t pcg_matvec(const cfd2d_poisson& op, const double* x, double* y, cudaStream_t s) {
    const int n = op.nx * op.ny;
    k_matvec<<<(n + 255) / 256, 256, 0, s>>>(op, x, y);
    return cudaGetLastError();
}

// Upper bound on the CTAs of the workspace solver on the current device (its partial
// arrays are sized for it): every SM times the most CTAs an SM can hold.
int max_grid_ctas() {
    const DevLimits d = dev_limits();
    return d.sms > 0 ? d.sms * kMaxCtasPerSm : 0;
}

size_t pcg_grid_workspace_doubles(int nx, int ny) {
    // R, P0, P1 (the slab form: boundary rows of z and p) + three partial arrays for
    // up to max_grid_ctas() CTAs (two used, as the parity sets of grid_sum) + barrier words
    return (size_t)3 * nx * ny + (size_t)3 * max_grid_ctas() * kSlot + 8;
}

template <bool VAR>
cudaError_t pcg_grid_launch_t(const PcgLaunch& L, cudaStream_t s) {
    const int n = L.op.nx * L.op.ny;
    const bool cl = L.op.grid_ctas == 16;
    if (L.op.grid_ctas != 0 && L.op.grid_ctas != -1 && L.op.grid_ctas != -2 && !cl) return cudaErrorInvalidValue;
    if (L.op.work == nullptr || L.op.work_bytes < pcg_grid_workspace_doubles(L.op.nx, L.op.ny) * sizeof(double))
        return cudaErrorInvalidValue;
    if constexpr (!VAR) {
        int Gs = 0, cap = 0;
        if ((L.op.grid_ctas == 0 || L.op.grid_ctas == -2) && !L.snap && slab_plan(L.op.nx, L.op.ny, &Gs, &cap)) {
            if (L.op.grid_ctas == -2) {
                switch (slab_cpt_for(cap)) {
                    case 1: return launch_slab<1, true>(L, Gs, cap, s);
                    case 2: return launch_slab<2, true>(L, Gs, cap, s);
                    case 4: return launch_slab<4, true>(L, Gs, cap, s);
                    default: return launch_slab<8, true>(L, Gs, cap, s);
                }
            }
            switch (slab_cpt_for(cap)) {
                case 1: return launch_slab<1, false>(L, Gs, cap, s);
                case 2: return launch_slab<2, false>(L, Gs, cap, s);
                case 4: return launch_slab<4, false>(L, Gs, cap, s);
                default: return launch_slab<8, false>(L, Gs, cap, s);
            }
        }
    }
    const int G = cl ? 16 : grid_blocks_for<VAR>(n);
    if (G < 1 || G > max_grid_ctas()) return cudaErrorInvalidConfiguration;
    PcgLaunch Lc = L;
    // the barrier words start from zero on every launch, whatever an earlier
    // launch that gave up on a wait left behind
    const size_t n3 = (size_t)3 * n + (size_t)3 * G * kSlot;
    cudaError_t e = cudaMemsetAsync(L.op.work + n3, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    if (cl) {
        // one 16-CTA cluster: its reductions use cluster barriers, so several such
        // solves (of different cases) can run side by side on the other SMs
        static bool configured[kMaxDevices];
        const DevLimits d = dev_limits();
        if (d.sms <= 0 || d.dev >= kMaxDevices) return cudaErrorInvalidDevice;
        if (!configured[d.dev]) {
            e = cudaFuncSetAttribute(k_pcg_grid<true, VAR>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
            configured[d.dev] = true;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16, 1, 1);
        cfg.blockDim = dim3(kClusterL2Threads, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 16;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, k_pcg_grid<true, VAR>, Lc);
    }
    void* args[] = {&Lc};
    return cudaLaunchCooperativeKernel((const void*)k_pcg_grid<false, VAR>, dim3(G), dim3(kGridThreads), args, 0,
                                       s);
}

cudaError_t pcg_grid_launch(const PcgLaunch& L, cudaStream_t s) {
    if (L.op.bx) {
        if (!L.op.by) return cudaErrorInvalidValue;
        return pcg_grid_launch_t<true>(L, s);
    }
    return pcg_grid_launch_t<false>(L, s);
}

// ---------------------------------------------------------------- launch
namespace {

size_t smem_bytes(int cap, bool var = false) {
    return (size_t)cap * ((kArrays + (var ? 4 : 0)) * sizeof(double) + 1) + 16;
}

// Kernel attributes are set once per instantiation and device, outside any stream
// capture (cfd2d_pcg_plan runs before the first launch): the maximum dynamic shared
// memory the hardware allows and permission for 16-CTA clusters.
template <class K>
cudaError_t configure_cluster_kernel(K kern, bool (&done)[kMaxDevices]) {
    const DevLimits d = dev_limits();
    if (d.sms <= 0 || d.dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (done[d.dev]) return cudaSuccess;
    const int dyn = d.smem_optin - (int)((32 * kMaxK + 2 * 16 * kMaxK + CFD2D_MAX_COMPONENTS) * sizeof(double)) - 1024;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    done[d.dev] = true;
    return cudaSuccess;
}

template <int CPT, bool PAIR, bool VAR = false>
cudaError_t configure_cpt() {
    static bool done[kMaxDevices];
    return configure_cluster_kernel(k_pcg_cluster<CPT, PAIR, VAR>, done);
}

template <int CPT, bool PAIR, bool VAR = false>
cudaError_t launch_cpt(const PcgLaunch& L, int C, cudaStream_t s) {
    auto kern = k_pcg_cluster<CPT, PAIR, VAR>;
    const size_t bytes = smem_bytes(L.cap_cells, VAR);
    cudaError_t e = configure_cpt<CPT, PAIR, VAR>();
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kPcgThreads, 1, 1);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, L);
}

// the single-reduction cluster form (k_pcg_cluster1): same attributes as configure_cpt
template <int CPT>
cudaError_t configure_cpt1() {
    static bool done[kMaxDevices];
    return configure_cluster_kernel(k_pcg_cluster1<CPT>, done);
}

// whether the single-reduction form's extra rows fit beside the cluster layout
bool cluster1_fits(int cap, int ny) {
    const DevLimits d = dev_limits();
    if (d.sms <= 0) return false;
    const size_t dyn = (size_t)d.smem_optin - (32 * kMaxK + 2 * 16 * kMaxK + CFD2D_MAX_COMPONENTS) * sizeof(double) - 1024;
    return 2 * ny <= kHaloPer * kPcgThreads && smem_bytes1(cap, ny) <= dyn;
}

template <int CPT>
cudaError_t launch_cpt1(const PcgLaunch& L, int C, cudaStream_t s) {
    cudaError_t e = configure_cpt1<CPT>();
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kPcgThreads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes1(L.cap_cells, L.op.ny);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_pcg_cluster1<CPT>, L);
}

// the mixed-precision solver: x and b in FP64, seven FP32 arrays, the coupling bits
size_t smem_bytes_mixed(int cap) { return (size_t)cap * (2 * sizeof(double) + 7 * sizeof(float) + 1) + 16; }

template <int CPT>
cudaError_t launch_mixed(const PcgLaunch& L, int C, cudaStream_t s) {
    static bool done[kMaxDevices];
    {
        const cudaError_t e = configure_cluster_kernel(k_pcg_cluster_mixed<CPT>, done);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kPcgThreads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes_mixed(L.cap_cells);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_pcg_cluster_mixed<CPT>, L);
}

int cpt_for(int cap) {
    const int need = (cap + kPcgThreads - 1) / kPcgThreads;
    if (need <= 1) return 1;
    if (need <= 2) return 2;
    if (need <= 4) return 4;
    if (need <= 8) return 8;
    return 0;
}

}  // namespace

// Whether the on-chip solver holds the variable-coefficient operator of an nx x ny
// grid on C CTAs (ny even: the paired-cell form; at most 4 cell pairs per thread).
bool pcg_var_cluster_fits(int nx, int ny, int C) {
    if (C < 1 || C > 16 || ny % 2 != 0) return false;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    const size_t dyn = (size_t)optin - (32 * kMaxK + 2 * 16 * kMaxK + CFD2D_MAX_COMPONENTS) * sizeof(double) - 1024;
    const int cap = ((nx + C - 1) / C) * ny;
    return smem_bytes(cap, true) <= dyn && cpt_for((cap + 1) / 2) != 0 && cpt_for((cap + 1) / 2) <= 4;
}

// Max cells one CTA can hold for a given dynamic shared-memory budget.
int pcg_cluster_capacity(size_t smem_limit) {
    return (int)((smem_limit - 16) / (kArrays * sizeof(double) + 1));
}

// Pick the cluster size for an nx x ny grid: smallest C (power of two, <= 16)
// whose slabs fit in shared memory and can be co-scheduled. 0 if none.
int pcg_cluster_plan(int nx, int ny) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    int smem_optin = 0;
    if (cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    // leave room for the static shared arrays of the kernel
    const size_t budget = (size_t)smem_optin - (32 * kMaxK + 2 * 16 * kMaxK + CFD2D_MAX_COMPONENTS) * sizeof(double) - 1024;
    const int capmax = pcg_cluster_capacity(budget);
    // target ~ 2-4 cells per thread before growing the cluster: fewer CTAs mean
    // cheaper barriers, and on-chip state is the point
    // smallest cluster whose slabs hold <= 4 cells per thread; else <= 8 per thread
    for (int pass = 0; pass < 2; ++pass) {
    for (int C = 1; C <= 16; C *= 2) {
        if (nx < C) break;
        const int rows = (nx + C - 1) / C;
        const long long cells = (long long)rows * ny;
        const long long lim = pass == 0 ? 4LL * kPcgThreads : 8LL * kPcgThreads;
        if (cells > capmax || cells > lim) continue;
        // co-scheduling check
        const int cpt = cpt_for((int)cells);
        if (!cpt) continue;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(C, 1, 1);
        cfg.blockDim = dim3(kPcgThreads, 1, 1);
        cfg.dynamicSmemBytes = smem_bytes((int)cells);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        cudaError_t e = cudaSuccess;
        const void* f = nullptr;
        switch (cpt) {
            case 1: e = configure_cpt<1, false>(); f = (const void*)k_pcg_cluster<1, false, false>; break;
            case 2: e = configure_cpt<2, false>(); f = (const void*)k_pcg_cluster<2, false, false>; break;
            case 4: e = configure_cpt<4, false>(); f = (const void*)k_pcg_cluster<4, false, false>; break;
            default: e = configure_cpt<8, false>(); f = (const void*)k_pcg_cluster<8, false, false>; break;
        }
        // the paired variant (even ny) has the same block size and shared memory; its
        // single-reduction form is configured here too (attributes before any capture)
        if (e == cudaSuccess) {
            switch (cpt_for((int)((cells + 1) / 2))) {
                case 1: e = configure_cpt<1, true>(); if (e == cudaSuccess) e = configure_cpt1<1>(); break;
                case 2: e = configure_cpt<2, true>(); if (e == cudaSuccess) e = configure_cpt1<2>(); break;
                case 4: e = configure_cpt<4, true>(); if (e == cudaSuccess) e = configure_cpt1<4>(); break;
                default: e = configure_cpt<8, true>(); if (e == cudaSuccess) e = configure_cpt1<8>(); break;
            }
        }
        if (e != cudaSuccess) { cudaGetLastError(); continue; }
        e = cudaOccupancyMaxActiveClusters(&nclusters, f, &cfg);
        if (e != cudaSuccess) { cudaGetLastError(); continue; }
        if (nclusters >= 1) return C;
    }
    }
    return 0;
}

cudaError_t pcg_launch(const PcgLaunch& L0, cudaStream_t s) {
    PcgLaunch L = L0;
    const int C = L.op.cluster;
    if (C == 0) return pcg_grid_launch(L, s);
    if (C < 1 || C > 16) return cudaErrorInvalidValue;
    const int rows = (L.op.nx + C - 1) / C;
    L.cap_cells = rows * L.op.ny;
    if (L.op.bx) {
        // variable coefficients: four more arrays per cell (pcg_var_cluster_fits)
        if (!L.op.by || L.op.mixed || L.op.ny % 2 != 0) return cudaErrorInvalidValue;
        switch (cpt_for((L.cap_cells + 1) / 2)) {
            case 1: return launch_cpt<1, true, true>(L, C, s);
            case 2: return launch_cpt<2, true, true>(L, C, s);
            case 4: return launch_cpt<4, true, true>(L, C, s);
            default: return cudaErrorInvalidValue;
        }
    }
    if (L.op.mixed) {
        // the cluster planned for the FP64 solver holds the 45-byte cells as well
        switch (cpt_for(L.cap_cells)) {
            case 1: return launch_mixed<1>(L, C, s);
            case 2: return launch_mixed<2>(L, C, s);
            case 4: return launch_mixed<4>(L, C, s);
            case 8: return launch_mixed<8>(L, C, s);
            default: return cudaErrorInvalidValue;
        }
    }
    if (L.op.ny % 2 == 0 && L.op.grid_ctas == -2 && cluster1_fits(L.cap_cells, L.op.ny)) {
        // the single-reduction form (opt-in; the default keeps scipy's two reductions)
        switch (cpt_for((L.cap_cells + 1) / 2)) {
            case 1: return launch_cpt1<1>(L, C, s);
            case 2: return launch_cpt1<2>(L, C, s);
            case 4: return launch_cpt1<4>(L, C, s);
            case 8: return launch_cpt1<8>(L, C, s);
            default: return cudaErrorInvalidValue;
        }
    }
    if (L.op.ny % 2 == 0) {
        switch (cpt_for((L.cap_cells + 1) / 2)) {
            case 1: return launch_cpt<1, true>(L, C, s);
            case 2: return launch_cpt<2, true>(L, C, s);
            case 4: return launch_cpt<4, true>(L, C, s);
            case 8: return launch_cpt<8, true>(L, C, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (cpt_for(L.cap_cells)) {
        case 1: return launch_cpt<1, false>(L, C, s);
        case 2: return launch_cpt<2, false>(L, C, s);
        case 4: return launch_cpt<4, false>(L, C, s);
        case 8: return launch_cpt<8, false>(L, C, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cfd
