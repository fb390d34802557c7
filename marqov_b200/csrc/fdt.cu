// Per-EMCS samples kept on the device, and the fluctuation-dissipation
// gradients of scalar phi^4 observables computed from them.
//
// Samples: after each EMCS the raw lattice sums of the measurement slot --
// interaction sum I = sum_i s_i sum_{j in nbrs(i)} s_j (every bond twice),
// M = sum_i s_i, Q2 = sum_i s_i^2, Q4 = sum_i (s_i^2 - 1)^2 -- are written as
// four FP64 values to a caller-owned device buffer (no host round trip).
//
// phi^4 in the reference's form (src/hamiltonian/Phi4.h:84-121, mass m):
//   S = beta H = -beta sum_<ij> phi_i phi_j + sum_i [m phi_i^2 + lambda (phi_i^2 - 1)^2]
// with per-sample observables
//   E  = H / N = (-I/2 + (m/beta) Q2 + (lambda/beta) Q4) / N,
//   |m| = |M| / N,  m2 = (M/N)^2,  m4 = m2^2,  U4 = 1 - <m4> / (3 <m2>^2).
// For theta in {beta, lambda}:  d<O>/dtheta = -cov(O, dS/dtheta) + <dO/dtheta>,
//   dS/dbeta = -I/2,  dS/dlambda = Q4,
//   dE/dbeta = -(m Q2 + lambda Q4) / (beta^2 N),  dE/dlambda = Q4 / (beta N),
// and dU4 = -d<m4> / (3 <m2>^2) + 2 <m4> d<m2> / (3 <m2>^3).
// Means and covariances are two-pass FP64 reductions, one CTA per replica.
#include <cuda_runtime.h>

#include "engine.h"

namespace mqv {

// acc slots (int64 for integer models, FP64 for float models) -> samples
__global__ void acc_to_samples(const long long* __restrict__ acc, int is_f32, int nslots, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    const long long* a = acc + (size_t)k * kAccStride;
    if (is_f32) {
        const double* d = reinterpret_cast<const double*>(a);
        out[4 * k + 0] = d[kAccEne];
        out[4 * k + 1] = d[kAccMag];
        out[4 * k + 2] = d[kAccSq];
        out[4 * k + 3] = d[kAccQ4];
    } else {
        out[4 * k + 0] = (double)a[kAccEne];
        out[4 * k + 1] = (double)a[kAccMag];
        out[4 * k + 2] = (double)a[kAccSq];
        out[4 * k + 3] = 0.0;
    }
}

cudaError_t launch_acc_to_samples(const long long* acc, int is_f32, int nslots, double* out, cudaStream_t st)
{
    acc_to_samples<<<(nslots + 127) / 128, 128, 0, st>>>(acc, is_f32, nslots, out);
    return cudaGetLastError();
}

struct Phi4Sample {
    double E, am, m2, m4, dSb, dSl, dEb, dEl;
};

__device__ __forceinline__ Phi4Sample phi4_sample(const double* __restrict__ s, double invN, double beta, double lam,
                                                  double mass)
{
    const double I = s[0], M = s[1], Q2 = s[2], Q4 = s[3];
    Phi4Sample o;
    o.E = (-0.5 * I + (mass / beta) * Q2 + (lam / beta) * Q4) * invN;
    o.am = fabs(M) * invN;
    o.m2 = o.am * o.am;
    o.m4 = o.m2 * o.m2;
    o.dSb = -0.5 * I;
    o.dSl = Q4;
    o.dEb = -(mass * Q2 + lam * Q4) / (beta * beta) * invN;
    o.dEl = Q4 / beta * invN;
    return o;
}

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (*red)[32])
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][wid] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = 0;
        for (int w = 0; w < nw; ++w) x += red[k][w];
        v[k] = x;
    }
    __syncthreads();
}

// samples: [nrep][nsamp][4]; obs: [nrep][3] (<E>, <|m|>, U4); jac: [nrep][3][2]
// (d/dbeta, d/dlambda); if gout ([nrep][3]) is given, grads receives
// [nrep][2] = gout . jac.
__global__ void phi4_fdt(const double* __restrict__ samples, int nsamp, double invN, const double* __restrict__ beta,
                         const double* __restrict__ lam, double mass, double* __restrict__ obs,
                         double* __restrict__ jac, const double* __restrict__ gout, double* __restrict__ grads)
{
    __shared__ double red[8][32];
    const int r = blockIdx.x;
    const double b = beta[r], l = lam[r];
    const double* s = samples + (size_t)r * nsamp * 4;
    // pass 1: means
    double mu[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < nsamp; k += blockDim.x) {
        const Phi4Sample p = phi4_sample(s + 4 * (size_t)k, invN, b, l, mass);
        mu[0] += p.E;
        mu[1] += p.am;
        mu[2] += p.m2;
        mu[3] += p.m4;
        mu[4] += p.dSb;
        mu[5] += p.dSl;
        mu[6] += p.dEb;
        mu[7] += p.dEl;
    }
    block_sum(mu, red);
#pragma unroll
    for (int k = 0; k < 8; ++k) mu[k] /= (double)nsamp;
    // pass 2: covariances of (E, |m|, m2, m4) with (dS/dbeta, dS/dlambda)
    double cv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < nsamp; k += blockDim.x) {
        const Phi4Sample p = phi4_sample(s + 4 * (size_t)k, invN, b, l, mass);
        const double db = p.dSb - mu[4], dl = p.dSl - mu[5];
        const double o[4] = {p.E - mu[0], p.am - mu[1], p.m2 - mu[2], p.m4 - mu[3]};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            cv[2 * j] += o[j] * db;
            cv[2 * j + 1] += o[j] * dl;
        }
    }
    block_sum(cv, red);
    if (threadIdx.x == 0) {
        double d[4][2];
        for (int j = 0; j < 4; ++j) {
            d[j][0] = -cv[2 * j] / (double)nsamp;
            d[j][1] = -cv[2 * j + 1] / (double)nsamp;
        }
        d[0][0] += mu[6];  // direct dE/dtheta
        d[0][1] += mu[7];
        const double m2 = mu[2], m4 = mu[3];
        const double u4 = 1.0 - m4 / (3.0 * m2 * m2);
        double du[2];
        for (int t = 0; t < 2; ++t) du[t] = -d[3][t] / (3.0 * m2 * m2) + 2.0 * m4 * d[2][t] / (3.0 * m2 * m2 * m2);
        double* ob = obs + 3 * (size_t)r;
        ob[0] = mu[0];
        ob[1] = mu[1];
        ob[2] = u4;
        double* jc = jac + 6 * (size_t)r;
        jc[0] = d[0][0];
        jc[1] = d[0][1];
        jc[2] = d[1][0];
        jc[3] = d[1][1];
        jc[4] = du[0];
        jc[5] = du[1];
        if (gout && grads) {
            const double* g = gout + 3 * (size_t)r;
            grads[2 * r + 0] = g[0] * jc[0] + g[1] * jc[2] + g[2] * jc[4];
            grads[2 * r + 1] = g[0] * jc[1] + g[1] * jc[3] + g[2] * jc[5];
        }
    }
}

cudaError_t launch_phi4_fdt(const double* samples, int nrep, int nsamp, double invN, const double* beta,
                            const double* lam, double mass, double* obs, double* jac, const double* gout,
                            double* grads, cudaStream_t st)
{
    phi4_fdt<<<nrep, 256, 0, st>>>(samples, nsamp, invN, beta, lam, mass, obs, jac, gout, grads);
    return cudaGetLastError();
}

}  // namespace mqv
