// Batched form: many independent domains (ensemble members or served
// requests) of uneven nx x ny x nz advance together.  One step is five
// launches whatever the number of members, captured once in a CUDA graph:
//   k_batch_forcing  relaxation-zone update of every forced species
//   k_batch_prep     species-independent per-step fields of every member
//   k_batch_upwind   donor-cell pass of every species of every member (a
//                    column march over shared-memory level planes per tile)
//   (counter reset)
//   k_batch_corr     persistent CTAs pulling (member, species, tile) items
//                    from a cost-sorted work list with an atomic counter and
//                    running the fused z-march of mpdata_fused.cuh on each.
// Member data lives in a device table (BatchMember); the simple kernels map
// their flat block index to a member by binary search over per-member block
// prefix sums.
#pragma once
#include "boundary_kernels.cuh"
#include "common.cuh"
#include "mpdata_fused.cuh"

namespace icar {

constexpr int BATCH_MAX_SPECIES = 32;

struct BatchMember {
    Geo g;
    float dx, dt;
    double dtd;
    int S, adv_den, nzone, pad;
    const float *u, *v, *w, *rho, *jac, *ju, *jv, *jw, *dz;
    float *Um, *Vm, *Wm, *Gc, *DJR, *Wp;
    const float *filter;
    const int *zone;
    const float *q0[BATCH_MAX_SPECIES];
    float *q1[BATCH_MAX_SPECIES];
    float *out[BATCH_MAX_SPECIES];
    float *forcing[BATCH_MAX_SPECIES];
    const float *dqdt[BATCH_MAX_SPECIES];
};

// index of the last prefix entry <= b (prefix[0] = 0, prefix[n] = total)
__device__ __forceinline__ int find_owner(const int *__restrict__ prefix, int n, int b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// pairs[p] = (member, species) of the p-th forced species; prefix over their
// blocks of ceil(nzone*nz/256).
__global__ void k_batch_forcing(const BatchMember *__restrict__ mem, const int *__restrict__ prefix,
                                const int2 *__restrict__ pairs, int npairs)
{
    const int p = find_owner(prefix, npairs, blockIdx.x);
    const int2 ms = pairs[p];
    const BatchMember &m = mem[ms.x];
    const size_t t = (size_t)(blockIdx.x - prefix[p]) * blockDim.x + threadIdx.x;
    const Geo g = m.g;
    if (t >= (size_t)m.nzone * g.nz) return;
    const int z = (int)(t % (size_t)m.nzone);
    const int k = (int)(t / (size_t)m.nzone);
    const int packed = m.zone[z];
    const int i = packed % g.nx, j = packed / g.nx;
    const size_t c = ix(g, i, k, j);
    float *q = const_cast<float *>(m.q0[ms.y]);
    float *fo = m.forcing[ms.y];
    const float fnew = (float)((double)fo[c] + (double)m.dqdt[ms.y][c] * m.dtd);
    fo[c] = fnew;
    const float flt = m.filter[packed];
    if (flt == 1.0f)
        q[c] = fnew;
    else if (flt < 1.0f)
        q[c] = (float)((double)q[c] + ((double)flt * m.dtd / 3600.0) * (double)(fnew - q[c]));
}

// prefix over members of ceil((nx+1)*nz*(ny+1)/256) blocks
__global__ void k_batch_prep(const BatchMember *__restrict__ mem, const int *__restrict__ prefix, int nmem)
{
    const int mi = find_owner(prefix, nmem, blockIdx.x);
    const BatchMember &m = mem[mi];
    const Geo g = m.g;
    const size_t t = (size_t)(blockIdx.x - prefix[mi]) * blockDim.x + threadIdx.x;
    const int ni = g.nx + 1, nk = g.nz, nj = g.ny + 1;
    const int i = (int)(t % (size_t)ni);
    const size_t rest = t / (size_t)ni;
    const int k = (int)(rest % (size_t)nk);
    const int j = (int)(rest / (size_t)nk);
    if (j >= nj) return;
    const int adv_den = m.adv_den;
    const float dt = m.dt, dx = m.dx;
    if (j < g.ny) {
        size_t c = ix(g, i, k, j);
        if (i >= 1 && i <= g.nx - 1) {
            float rr = adv_den ? m.rho[c] : 1.0f;
            float rl = adv_den ? m.rho[c - 1] : 1.0f;
            m.Um[c] = m.u[c] * dt * (rr + rl) * 0.5f * m.ju[c] / dx;
        } else {
            m.Um[c] = 0.0f;
        }
        if (i < g.nx) {
            float r0 = adv_den ? m.rho[c] : 1.0f;
            float wm;
            if (k < g.nz - 1) {
                float r1 = adv_den ? m.rho[ix(g, i, k + 1, j)] : 1.0f;
                wm = m.w[c] * dt * m.jw[c] * (r1 + r0) * 0.5f;
            } else {
                wm = m.w[c] * dt * m.jw[c] * r0;
            }
            m.Wm[c] = wm;
            const float d = m.dz[c], jj = m.jac[c], rh = m.rho[c];
            m.Gc[c] = jj * rh;
            m.DJR[c] = d * jj * rh;
            m.Wp[c] = wm / d;
        }
    }
    if (i < g.nx) {
        size_t c = ix(g, i, k, j);
        if (j >= 1 && j <= g.ny - 1) {
            float rr = adv_den ? m.rho[c] : 1.0f;
            float rl = adv_den ? m.rho[ix(g, i, k, j - 1)] : 1.0f;
            m.Vm[c] = m.v[c] * dt * (rr + rl) * 0.5f * m.jv[c] / dx;
        } else {
            m.Vm[c] = 0.0f;
        }
    }
}

// Donor-cell pass of every member: prefix over members of
// upwind_cols_blocks(g, S, sg) blocks, each one 32 x 8 column tile of one
// species group (upwind_cols_tile of mpdata_fused.cuh).
__host__ __device__ inline int upwind_cols_group(int S, int sg) { return min(upwind_group(S, sg), upf::SGMAX); }
__host__ __device__ inline int upwind_cols_blocks(const Geo &g, int S, int sg)
{
    const int grp = upwind_cols_group(S, sg);
    const int ng = grp > 0 ? (S + grp - 1) / grp : 0;
    return ng * ((g.nx + upf::BX - 1) / upf::BX) * ((g.ny + upf::BY - 1) / upf::BY);
}

__global__ void __launch_bounds__(upf::NT)
    k_batch_upwind(const BatchMember *__restrict__ mem, const int *__restrict__ prefix, int nmem, int sg)
{
    extern __shared__ float4 sm4[];
    const int mi = find_owner(prefix, nmem, blockIdx.x);
    const BatchMember &m = mem[mi];
    const Geo g = m.g;
    const int grp = upwind_cols_group(m.S, sg);
    const int tx = (g.nx + upf::BX - 1) / upf::BX, ty = (g.ny + upf::BY - 1) / upf::BY;
    const int local = blockIdx.x - prefix[mi];
    const int s0 = (local / (tx * ty)) * grp, tile = local % (tx * ty);
    upwind_cols_tile(reinterpret_cast<float *>(sm4), g, m.q0 + s0, m.q1 + s0, m.out + s0, min(grp, m.S - s0),
                     (tile % tx) * upf::BX, (tile / tx) * upf::BY, m.Um, m.Vm, m.Wm, m.Gc, m.DJR);
}

// Persistent correction kernel: items are (member, species, i0, j0).
template <bool FCT, class SH>
__global__ void __launch_bounds__(SH::NT, (SH::NT <= 128 ? 5 : SH::NT <= 256 ? 3 : SH::NT <= 512 ? 2 : 1))
    k_batch_corr(const BatchMember *__restrict__ mem, const int4 *__restrict__ items, int n_items,
                 int *__restrict__ counter)
{
    extern __shared__ float4 sm4[];
    __shared__ int next;
    float *sm = reinterpret_cast<float *>(sm4);
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1);
        __syncthreads();
        const int it = next;
        __syncthreads();
        if (it >= n_items) break;
        const int4 w = items[it];
        const BatchMember &m = mem[w.x];
        mp_corr_tile<FCT, SH>(sm, m.g, m.q0[w.y], m.q1[w.y], m.out[w.y], w.z, w.w, m.Um, m.Vm, m.Wp, m.Gc,
                              m.DJR, m.dz);
    }
}

template <class SH>
inline cudaError_t batch_corr_attr()
{
    cudaError_t e = cudaFuncSetAttribute(k_batch_corr<true, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mpf::smem_bytes<SH>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_corr<false, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mpf::smem_bytes<SH>());
    return e;
}

inline cudaError_t batch_setup()
{
    cudaError_t e = cudaFuncSetAttribute(k_batch_upwind, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upf::SMEM);
    if (e == cudaSuccess) e = batch_corr_attr<MpShape8>();
    if (e == cudaSuccess) e = batch_corr_attr<MpShape16>();
    if (e == cudaSuccess) e = batch_corr_attr<MpShape24>();
    if (e == cudaSuccess) e = batch_corr_attr<MpShape32>();
    return e;
}

// CTAs of the persistent kernel that fit on the device at once.
template <class SH>
inline int batch_corr_ctas(int fct, int nsm)
{
    int per = 0;
    if (fct)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_corr<true, SH>, SH::NT, mpf::smem_bytes<SH>());
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_corr<false, SH>, SH::NT, mpf::smem_bytes<SH>());
    return (per > 0 ? per : 1) * nsm;
}

template <class SH>
inline void batch_corr_launch_t(cudaStream_t st, int ctas, int fct, const BatchMember *mem, const int4 *items,
                                int n, int *counter)
{
    if (fct)
        k_batch_corr<true, SH><<<ctas, SH::NT, mpf::smem_bytes<SH>(), st>>>(mem, items, n, counter);
    else
        k_batch_corr<false, SH><<<ctas, SH::NT, mpf::smem_bytes<SH>(), st>>>(mem, items, n, counter);
}

inline int batch_corr_max_ctas(int shape, int fct, int nsm)
{
    switch (shape) {
    case 0: return batch_corr_ctas<MpShape8>(fct, nsm);
    case 2: return batch_corr_ctas<MpShape24>(fct, nsm);
    case 3: return batch_corr_ctas<MpShape32>(fct, nsm);
    default: return batch_corr_ctas<MpShape16>(fct, nsm);
    }
}

inline void batch_corr_launch(cudaStream_t st, int shape, int ctas, int fct, const BatchMember *mem,
                              const int4 *items, int n, int *counter)
{
    switch (shape) {
    case 0: batch_corr_launch_t<MpShape8>(st, ctas, fct, mem, items, n, counter); break;
    case 2: batch_corr_launch_t<MpShape24>(st, ctas, fct, mem, items, n, counter); break;
    case 3: batch_corr_launch_t<MpShape32>(st, ctas, fct, mem, items, n, counter); break;
    default: batch_corr_launch_t<MpShape16>(st, ctas, fct, mem, items, n, counter); break;
    }
}

}  // namespace icar
