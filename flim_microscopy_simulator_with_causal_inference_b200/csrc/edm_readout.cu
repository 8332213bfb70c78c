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

// One thread per pixel streams the pixel's row in 16-byte loads; the lanes
// of a warp read 32 rows side by side, and the next load of each lane hits
// the sector the previous one opened, so the stack is read from DRAM once.
// Intensity and sum n_k k are exact integer sums (sum n_k t_k =
// width * (sum n_k k + intensity / 2)); the phasor sums are float64.
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
    for (int q = 0; q < nq; ++q) {
      const uint4 v = __ldg(row + q);
      const uint32_t n4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = 4 * q + i;
        I += n4[i];
        KW += (uint64_t)n4[i] * (uint64_t)k;
        const double n = (double)n4[i];
        G += n * c_k[k];
        S += n * s_k[k];
      }
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
