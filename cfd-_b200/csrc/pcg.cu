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

constexpr int kPcgThreads = 1024;
constexpr int kSlot = 4 + CFD2D_MAX_COMPONENTS;  // doubles per reduction slot

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

// cluster-wide sum of K per-thread values: block tree, then the C CTA partials
// added in rank order by every CTA. Returns the same value in every thread.
template <int K>
__device__ __forceinline__ void cluster_sum(cg::cluster_group& cluster, double (&v)[K],
                                            double* red_smem, double* slot, int C) {
    block_sum<K>(v, red_smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) slot[k] = v[k];
    }
    cluster.sync();
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = 0.0;
        if (lane < C) x = cluster.map_shared_rank(slot, lane)[k];
        // fixed-shape tree over the (at most 16) partials
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[k] = x;
    }
}

}  // namespace

template <int CPT>
__global__ void __launch_bounds__(kPcgThreads, 1) k_pcg_cluster(PcgLaunch L) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int me = (int)cluster.block_rank();
    if (L.active && *L.active == 0) return;  // uniform over the cluster

    const cfd2d_poisson& op = L.op;
    const int nx = op.nx, ny = op.ny;
    const bool periodic = op.periodic != 0;
    const int r0 = row0_of(me, nx, C), r1 = row0_of(me + 1, nx, C);
    const int nloc = (r1 - r0) * ny;
    const int cap = L.cap_cells;
    const int tid = threadIdx.x;
    const double mdx2 = -op.dx2, mdy2 = -op.dy2;

    extern __shared__ __align__(16) double sm[];
    double* X = sm;
    double* R = X + cap;
    double* P0 = R + cap;
    double* P1 = P0 + cap;
    double* DI = P1 + cap;
    double* DG = DI + cap;
    uint8_t* NB = reinterpret_cast<uint8_t*>(DG + cap);
    __shared__ double red_smem[32 * kSlot];
    __shared__ double slotA[kSlot];
    __shared__ double slotB[kSlot];

    // ------------------------------------------------------------ prologue: load
    const int ncomp = op.ncomp;
    double dt = 1.0;
    if (L.rhs_mode == 1) dt = L.dt_ptr ? *L.dt_ptr : L.dt_const;
    double csum[CFD2D_MAX_COMPONENTS + 1];
#pragma unroll
    for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) csum[k] = 0.0;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int i = r0 + c / ny, j = c % ny;
        const int gidx = i * ny + j;
        const uint8_t nb = op.nbr[gidx];
        NB[c] = nb;
        X[c] = op.x0[gidx];
        DI[c] = op.dinv[gidx];
        DG[c] = op.diag[gidx];
        double braw = 0.0;
        if (nb & 0x80) {
            if (L.rhs_mode == 0) {
                braw = L.rhs[gidx];
            } else {
                // div(F, G) / dt at interior cell (i+1, j+1) (cfd2d/solver.py:264-266)
                const int pu = ny + 2, pv = ny + 1;
                const int ig = i + 1, jg = j + 1;
                const double div = (L.F[ig * pu + jg] - L.F[(ig - 1) * pu + jg]) / L.dx +
                                   (L.G[ig * pv + jg] - L.G[ig * pv + jg - 1]) / L.dy;
                braw = div / dt;
            }
            const int lab = op.label[gidx];
            if (lab >= 0 && lab < CFD2D_MAX_COMPONENTS) {
#pragma unroll
                for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                    if (k == lab) csum[k] += braw;
            }
            if (X[c] != 0.0) csum[CFD2D_MAX_COMPONENTS] += 1.0;
        }
        R[c] = braw;
    }
    // component sums of b (mean removal, cfd2d/pressure.py:155-160) and "x0.any()"
    {
        double v[CFD2D_MAX_COMPONENTS + 1];
#pragma unroll
        for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) v[k] = csum[k];
        cluster_sum<CFD2D_MAX_COMPONENTS + 1>(cluster, v, red_smem, slotA, C);
#pragma unroll
        for (int k = 0; k <= CFD2D_MAX_COMPONENTS; ++k) csum[k] = v[k];
    }
    const bool x_any = csum[CFD2D_MAX_COMPONENTS] > 0.0;

    // b = -(b_raw - mean), r = b - A x0 (only if x0 has a nonzero), norms
    double part[3] = {0.0, 0.0, 0.0};
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const uint8_t nb = NB[c];
        if (!(nb & 0x80)) { P1[c] = 0.0; P0[c] = 0.0; R[c] = 0.0; continue; }
        const int i = r0 + c / ny, j = c % ny;
        const int gidx = i * ny + j;
        double b = R[c];
        const int lab = op.label[gidx];
        if (lab >= 0) {
            double mean = 0.0;
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) mean = csum[k] / op.comp_count[k];
            b = b - mean;
        }
        b = -b;
        P1[c] = b;  // kept for the ||b|| == 0 return
        double r = b;
        if (x_any) {
            double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
            if (nb & 2) tS = mdy2 * X[c - 1];
            if (nb & 4) tN = mdy2 * X[c + 1];
            if (nb & 1) {
                const int iw = (i == 0) ? nx - 1 : i - 1;
                const double* row = (iw >= r0 && iw < r1)
                                        ? X + (iw - r0) * ny
                                        : cluster.map_shared_rank(X, owner_of(iw, nx, C)) +
                                              (iw - row0_of(owner_of(iw, nx, C), nx, C)) * ny;
                tW = mdx2 * row[j];
            }
            if (nb & 8) {
                const int ie = (i == nx - 1) ? 0 : i + 1;
                const double* row = (ie >= r0 && ie < r1)
                                        ? X + (ie - r0) * ny
                                        : cluster.map_shared_rank(X, owner_of(ie, nx, C)) +
                                              (ie - row0_of(owner_of(ie, nx, C), nx, C)) * ny;
                tE = mdx2 * row[j];
            }
            const double ax = row_sum(periodic, i, nx, tW, tS, DG[c] * X[c], tN, tE);
            r = b - ax;
        }
        // R is only read by other CTAs inside the iteration loop, after the
        // barrier of the reduction below; X (read here across CTAs) is unchanged
        R[c] = r;
        P0[c] = 0.0;
        part[0] += b * b;
        part[1] += r * r;
        part[2] += r * (DI[c] * r);
    }
    cluster_sum<3>(cluster, part, red_smem, slotB, C);
    const double bnrm2 = sqrt(part[0]);
    double rr = part[1];
    double rho = part[2];  // r . (M r) for the first iteration
    const double atol = L.rtol * bnrm2;
    int it = 0;
    bool converged = false;
    if (bnrm2 == 0.0) {
        // scipy returns b itself
        for (int c = tid; c < nloc; c += kPcgThreads) X[c] = P1[c];
        converged = true;
    } else {
        double beta = 0.0;
        int cur = 0;  // p of this iteration goes to buffer cur
        double q[CPT];
        for (it = 0; it < L.maxiter; ++it) {
            if (sqrt(rr) < atol) { converged = true; break; }
            double* Pn = cur ? P1 : P0;  // new p
            const double* Po = cur ? P0 : P1;  // previous p
            const bool first = (it == 0);
            double pq = 0.0;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                q[k] = 0.0;
                const int c = tid + k * kPcgThreads;
                if (c >= nloc) continue;
                const uint8_t nb = NB[c];
                if (!(nb & 0x80)) continue;
                const int i = r0 + c / ny, j = c % ny;
                // p_new = beta * p_old + dinv * r at a cell with local arrays po/rr_/di
#define PNEW(po, r_, di, idx) (first ? ((di)[idx] * (r_)[idx]) : ((po)[idx] * beta + (di)[idx] * (r_)[idx]))
                const double pC = PNEW(Po, R, DI, c);
                double tW = 0.0, tS = 0.0, tN = 0.0, tE = 0.0;
                if (nb & 2) tS = mdy2 * PNEW(Po, R, DI, c - 1);
                if (nb & 4) tN = mdy2 * PNEW(Po, R, DI, c + 1);
                if (nb & 1) {
                    const int iw = (i == 0) ? nx - 1 : i - 1;
                    if (iw >= r0 && iw < r1) {
                        const int o = (iw - r0) * ny + j;
                        tW = mdx2 * PNEW(Po, R, DI, o);
                    } else {
                        const int ow = owner_of(iw, nx, C);
                        const int o = (iw - row0_of(ow, nx, C)) * ny + j;
                        const double* po = cluster.map_shared_rank(Po, ow);
                        const double* rr_ = cluster.map_shared_rank(R, ow);
                        const double* di = cluster.map_shared_rank(DI, ow);
                        tW = mdx2 * PNEW(po, rr_, di, o);
                    }
                }
                if (nb & 8) {
                    const int ie = (i == nx - 1) ? 0 : i + 1;
                    if (ie >= r0 && ie < r1) {
                        const int o = (ie - r0) * ny + j;
                        tE = mdx2 * PNEW(Po, R, DI, o);
                    } else {
                        const int oe = owner_of(ie, nx, C);
                        const int o = (ie - row0_of(oe, nx, C)) * ny + j;
                        const double* po = cluster.map_shared_rank(Po, oe);
                        const double* rr_ = cluster.map_shared_rank(R, oe);
                        const double* di = cluster.map_shared_rank(DI, oe);
                        tE = mdx2 * PNEW(po, rr_, di, o);
                    }
                }
#undef PNEW
                const double qq = row_sum(periodic, i, nx, tW, tS, DG[c] * pC, tN, tE);
                Pn[c] = pC;
                q[k] = qq;
                pq += pC * qq;
            }
            {
                double v[1] = {pq};
                cluster_sum<1>(cluster, v, red_smem, slotA, C);
                pq = v[0];
            }
            const double alpha = rho / pq;
            double v2[2] = {0.0, 0.0};
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int c = tid + k * kPcgThreads;
                if (c >= nloc) continue;
                if (!(NB[c] & 0x80)) continue;
                X[c] = X[c] + alpha * Pn[c];
                const double r = R[c] - alpha * q[k];
                R[c] = r;
                v2[0] += r * r;
                v2[1] += r * (DI[c] * r);
            }
            cluster_sum<2>(cluster, v2, red_smem, slotB, C);
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
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int i = r0 + c / ny, j = c % ny;
        const int gidx = i * ny + j;
        const double x = X[c];
        op.x0[gidx] = x;
        if (ncomp > 0 && (NB[c] & 0x80)) {
            const int lab = op.label[gidx];
#pragma unroll
            for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                if (k == lab) xs[k] += x;
        }
    }
    if (ncomp > 0) cluster_sum<CFD2D_MAX_COMPONENTS>(cluster, xs, red_smem, slotA, C);
    const int pp = ny + 2;
    for (int c = tid; c < nloc; c += kPcgThreads) {
        const int i = r0 + c / ny, j = c % ny;
        const int gidx = i * ny + j;
        double pv = 0.0;
        if (NB[c] & 0x80) {
            pv = X[c];
            const int lab = op.label[gidx];
            if (lab >= 0) {
                double mean = 0.0;
#pragma unroll
                for (int k = 0; k < CFD2D_MAX_COMPONENTS; ++k)
                    if (k == lab) mean = xs[k] / op.comp_count[k];
                pv = pv - mean;
            }
        }
        if (!L.p_padded) {
            L.p_out[gidx] = pv;
        } else {
            L.p_out[(i + 1) * pp + j + 1] = pv;
            // periodic ghost rows: p[0,:] = p[nx,:], p[nx+1,:] = p[1,:]
            if (periodic && i == nx - 1) L.p_out[0 * pp + j + 1] = pv;
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
            for (int j = tid; j < pp; j += kPcgThreads) {
                if (!periodic || j == 0 || j == ny + 1) L.p_out[j] = 0.0;
            }
        }
        if (me == C - 1) {
            for (int j = tid; j < pp; j += kPcgThreads) {
                if (!periodic || j == 0 || j == ny + 1) L.p_out[(nx + 1) * pp + j] = 0.0;
            }
        }
    }
    if (me == 0 && tid == 0) {
        if (L.iters_out) *L.iters_out = it;
        if (L.iters_out2) *L.iters_out2 = it;
        if (L.status_out && !converged) atomicOr(L.status_out, CFD2D_S_CG_MAXITER);
    }
    // keep every CTA's shared memory alive until all remote readers are done
    cluster.sync();
}

// ---------------------------------------------------------------- launch
namespace {

size_t smem_bytes(int cap) { return (size_t)cap * (6 * sizeof(double) + 1) + 16; }

// Kernel attributes are set once per instantiation, outside any stream capture
// (cfd2d_pcg_plan runs before the first launch): the maximum dynamic shared
// memory the hardware allows and permission for 16-CTA clusters.
template <int CPT>
cudaError_t configure_cpt() {
    static bool done = false;
    if (done) return cudaSuccess;
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const int dyn = optin - (int)((32 * kSlot + 2 * kSlot) * sizeof(double)) - 1024;
    e = cudaFuncSetAttribute(k_pcg_cluster<CPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_pcg_cluster<CPT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    done = true;
    return cudaSuccess;
}

template <int CPT>
cudaError_t launch_cpt(const PcgLaunch& L, int C, cudaStream_t s) {
    auto kern = k_pcg_cluster<CPT>;
    const size_t bytes = smem_bytes(L.cap_cells);
    cudaError_t e = configure_cpt<CPT>();
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

int cpt_for(int cap) {
    const int need = (cap + kPcgThreads - 1) / kPcgThreads;
    if (need <= 1) return 1;
    if (need <= 2) return 2;
    if (need <= 4) return 4;
    if (need <= 8) return 8;
    return 0;
}

}  // namespace

// Max cells one CTA can hold for a given dynamic shared-memory budget.
int pcg_cluster_capacity(size_t smem_limit) {
    return (int)((smem_limit - 16) / (6 * sizeof(double) + 1));
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
    const size_t budget = (size_t)smem_optin - (32 * kSlot + 2 * kSlot) * sizeof(double) - 1024;
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
            case 1: e = configure_cpt<1>(); f = (const void*)k_pcg_cluster<1>; break;
            case 2: e = configure_cpt<2>(); f = (const void*)k_pcg_cluster<2>; break;
            case 4: e = configure_cpt<4>(); f = (const void*)k_pcg_cluster<4>; break;
            default: e = configure_cpt<8>(); f = (const void*)k_pcg_cluster<8>; break;
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
    if (C < 1 || C > 16) return cudaErrorInvalidValue;
    const int rows = (L.op.nx + C - 1) / C;
    L.cap_cells = rows * L.op.ny;
    switch (cpt_for(L.cap_cells)) {
        case 1: return launch_cpt<1>(L, C, s);
        case 2: return launch_cpt<2>(L, C, s);
        case 4: return launch_cpt<4>(L, C, s);
        case 8: return launch_cpt<8>(L, C, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cfd
