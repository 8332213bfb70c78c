// edm_readout.cu — lifetime readouts of TCSPC stacks on the device.
//
// For every pixel of a uint32 stack [n_px][n_bins] (the engine's FLIM stacks
// or the batched acquisition's histograms), in float64:
//   intensity = sum_k n_k;
//   tau_mean  = sum_k n_k t_k / intensity, t_k = (k + 0.5) T / n_bins in ns,
//               NaN below min_counts_mean           (analysis.py:87-150);
//   g, s      = sum_k n_k cos(phi_k) / intensity, sum_k n_k sin(phi_k) / intensity,
//               phi_k = 2 pi h (k + 0.5) / n_bins, 0 below min_counts_phasor;
//   tau_phi   = (s / g) / omega, omega = 2 pi h / T in 1/ns, where g > 1e-10;
//   tau_mod   = sqrt(1 / m^2 - 1) / omega, m^2 = g^2 + s^2 in (1e-10, 1 - 1e-10)
//               (analysis.py:497-566); NaN elsewhere.
// The kernel streams the stack once.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/edm_b200.h"
#include "edm_error.h"

namespace {

// Exact float64 value of an integer v < 2^52: the double whose bits are
// 2^52 + v, minus 2^52 (one add instead of an integer-to-double conversion).
__device__ __forceinline__ double u52_to_f64(uint64_t v) {
  const double d = __hiloint2double(0x43300000 | (int)(uint32_t)(v >> 32), (int)(uint32_t)v);
  return __dsub_rn(d, 4503599627370496.0);
}

// Bins k and K-1-k share |cos| and |sin| of their phases (phi_{K-1-k} =
// 2 pi h - phi_k), so a pair adds (n_k + n_{K-1-k}) cos(phi_k) to G and
// (n_k - n_{K-1-k}) sin(phi_k) to S: two float64 multiply-adds per pair.
__device__ __forceinline__ void readout_pair(uint32_t na, uint32_t nb, int k, int kb, const double* c_k,
                                             const double* s_k, uint64_t& I, uint64_t& KW, double& G, double& S) {
  I += (uint64_t)na + nb;
  KW += (uint64_t)na * (uint32_t)k + (uint64_t)nb * (uint32_t)kb;
  G = fma(u52_to_f64((uint64_t)na + nb), c_k[k], G);
  S = fma(__dsub_rn(u52_to_f64((uint64_t)na + 4294967296ull - nb), 4294967296.0), s_k[k], S);
}

// One thread per pixel streams the pixel's row in 16-byte loads from both
// ends; the lanes of a warp read 32 rows side by side, so the stack is read
// from DRAM once.  Intensity and sum n_k k are exact integer sums (sum n_k
// t_k = width * (sum n_k k + intensity / 2)); the phasor sums are float64.
__global__ void __launch_bounds__(256) k_readout(const uint32_t* __restrict__ stack, int64_t n_px, int n_bins,
                                                 double T_ns, int harmonic, int min_mean, int min_phasor,
                                                 double* __restrict__ out) {
  __shared__ double c_k[256], s_k[256];
  for (int k = threadIdx.x; k < n_bins; k += blockDim.x) {
    const double phi = 2.0 * M_PI * harmonic * (k + 0.5) / n_bins;
    c_k[k] = cos(phi);
    s_k[k] = sin(phi);
  }
  __syncthreads();
  const int nq = n_bins / 4;  // uint4 per pixel
  const double width = T_ns / n_bins;
  const double omega = 2.0 * M_PI * harmonic / T_ns;
  const double nan = __longlong_as_double(0x7FF8000000000000ll);
  for (int64_t px = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; px < n_px; px += (int64_t)gridDim.x * blockDim.x) {
    const uint4* row = reinterpret_cast<const uint4*>(stack + px * (int64_t)n_bins);
    uint64_t I = 0, KW = 0;
    double G = 0.0, S = 0.0;
    int q = 0;
    for (; q < nq - 1 - q; ++q) {  // word q (bins 4q..4q+3) against word nq-1-q, reversed
      const int qb = nq - 1 - q;
      const uint4 a = __ldg(row + q), b = __ldg(row + qb);
      readout_pair(a.x, b.w, 4 * q, 4 * qb + 3, c_k, s_k, I, KW, G, S);
      readout_pair(a.y, b.z, 4 * q + 1, 4 * qb + 2, c_k, s_k, I, KW, G, S);
      readout_pair(a.z, b.y, 4 * q + 2, 4 * qb + 1, c_k, s_k, I, KW, G, S);
      readout_pair(a.w, b.x, 4 * q + 3, 4 * qb, c_k, s_k, I, KW, G, S);
    }
    if (q == nq - 1 - q) {  // odd word count: the middle word pairs within itself
      const uint4 a = __ldg(row + q);
      readout_pair(a.x, a.w, 4 * q, 4 * q + 3, c_k, s_k, I, KW, G, S);
      readout_pair(a.y, a.z, 4 * q + 1, 4 * q + 2, c_k, s_k, I, KW, G, S);
    }
    const double In = (double)I;
    const double tau = In >= min_mean ? width * ((double)KW + 0.5 * In) / In : nan;
    const bool mask = In >= min_phasor;
    const double g = mask ? G / In : 0.0, s = mask ? S / In : 0.0;
    const bool valid = mask && g > 1e-10;
    const double m2 = g * g + s * s;
    out[0 * n_px + px] = In;
    out[1 * n_px + px] = tau;
    out[2 * n_px + px] = g;
    out[3 * n_px + px] = s;
    out[4 * n_px + px] = valid ? (s / g) / omega : nan;
    out[5 * n_px + px] = (valid && m2 > 1e-10 && m2 < 1.0 - 1e-10) ? sqrt(1.0 / m2 - 1.0) / omega : nan;
  }
}

}  // namespace

extern "C" int edm_readout_lifetimes(const uint32_t* stack_dev, int64_t n_px, int32_t n_bins, double time_range_s,
                                     int32_t harmonic, int32_t min_counts_mean, int32_t min_counts_phasor,
                                     double* out_dev, void* stream) {
  if (!stack_dev || !out_dev || n_px < 0 || n_bins <= 0 || n_bins > 256 || n_bins % 4 != 0 || !(time_range_s > 0.0) ||
      harmonic < 1)
    return edm::report_error(EDM_EINVAL,
                             "edm_readout_lifetimes: bad argument (n_bins must be a multiple of 4 up to 256)");
  if (((uintptr_t)stack_dev & 15u) != 0)
    return edm::report_error(EDM_EINVAL, "edm_readout_lifetimes: stack must be 16-byte aligned");
  if (n_px == 0) return EDM_OK;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_readout, 256, 0);
  const int64_t want = (n_px + 255) / 256, cap = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  const unsigned blocks = (unsigned)(want < cap ? want : cap);
  k_readout<<<blocks, 256, 0, (cudaStream_t)stream>>>(stack_dev, n_px, n_bins, time_range_s * 1e9, harmonic,
                                                      min_counts_mean, min_counts_phasor, out_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return edm::report_error(EDM_ECUDA, std::string("edm_readout_lifetimes: ") + cudaGetErrorString(e));
  return EDM_OK;
}
