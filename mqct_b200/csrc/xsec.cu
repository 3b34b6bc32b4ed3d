// Cross sections on the device: INELAST_CALC (MQCT_SOURCE_CODES/propagator.f:4752-4851)
// from the amplitudes the propagation leaves in device memory, so that a batch's
// amplitudes need not travel to the host.
//
//   P_f(t)        = sum over the states s of channel f of |a_s(t)|^2      (per trajectory)
//   sigma_J,f     = pi / k^2 (2J+1)/(2j+1) sum_{l=|J-j|}^{J+j} P_f(traj(l)) a_bohr^2
//   sigma_f       = sum_J sigma_J,f
// with traj(l) = (l - L_MIN) / DL, the trajectory of l's bin (TRAJ_ORB,
// MQCT_SOURCE_CODES/propagator.f:5127-5134); sigma in Angstrom^2 as the reference
// prints it (PARTIAL_CROSS_SECTIONS_J.out, M_PROJ_CROSSECTIONS.out).
#include <cuda_runtime.h>

#include "common.cuh"
#include "mqct_b200.h"

namespace mqct {
namespace {

constexpr int kMaxChannels = 2048;
constexpr double kABohr = 0.52917721067;  // the a_bohr of INELAST_CALC

// First state of every channel (states of a channel are contiguous in the
// reference's channel-major order), passed by value: no device buffer needed.
struct ChannelRanges {
  int n;
  int first[kMaxChannels + 1];
};

// One CTA per trajectory; threads over channels; fixed summation order.
__global__ void channel_prob_kernel(const double* __restrict__ amp, int n_states,
                                   ChannelRanges ch, double* __restrict__ prob) {
  const int64_t t = blockIdx.x;
  const double* a = amp + (size_t)t * 2 * n_states;
  for (int c = threadIdx.x; c < ch.n; c += blockDim.x) {
    double p = 0.0;
    for (int s = ch.first[c]; s < ch.first[c + 1]; ++s) {
      const double re = a[s], im = a[n_states + s];
      p += re * re + im * im;
    }
    prob[(size_t)t * ch.n + c] = p;
  }
}

// One thread per (J, channel): the J-resolved cross section.
__global__ void partial_sigma_kernel(const double* __restrict__ prob, int64_t n_traj, int n_ch,
                                     int j_ini, int J_down, int n_J, int L_min, int dl,
                                     double k_vec, double* __restrict__ partial) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_J * n_ch) return;
  const int J = J_down + (int)(idx / n_ch), c = (int)(idx % n_ch);
  const double w = (2.0 * J + 1.0) / (k_vec * k_vec) / (2.0 * j_ini + 1) * kPi;
  double s = 0.0;
  const int l_lo = J - j_ini < 0 ? j_ini - J : J - j_ini;
  for (int l = l_lo; l <= J + j_ini; ++l) {
    const int64_t id = (l - L_min) / dl;
    if (l - L_min < 0 || id >= n_traj) continue;
    s += prob[id * n_ch + c] * w;
  }
  partial[idx] = s * kABohr * kABohr;
}

// One thread per channel: the sum over J in J order.
__global__ void sigma_kernel(const double* __restrict__ partial, int n_J, int n_ch,
                             double* __restrict__ sigma) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_ch) return;
  double s = 0.0;
  for (int J = 0; J < n_J; ++J) s += partial[(size_t)J * n_ch + c];
  sigma[c] = s;
}

}  // namespace
}  // namespace mqct

using namespace mqct;

extern "C" int mqct_cross_sections_device(const double* d_amp, int64_t n_traj, int32_t n_states,
                                          const int32_t* indx_chann, int32_t n_channels,
                                          int32_t j_ini, int32_t J_down, int32_t J_up,
                                          int32_t L_min, int32_t dl, double k_vec,
                                          double* d_prob, double* d_partial, double* d_sigma,
                                          void* stream) {
  MQCT_ARG_CHECK(d_amp && indx_chann && d_prob && d_partial && d_sigma, "null argument");
  MQCT_ARG_CHECK(n_traj > 0 && n_traj < ((int64_t)1 << 31) && n_states > 0, "bad sizes");
  MQCT_ARG_CHECK(n_channels > 0 && n_channels <= kMaxChannels,
                 "n_channels must be in 1..%d (got %d)", kMaxChannels, n_channels);
  MQCT_ARG_CHECK(j_ini >= 0 && J_down >= 0 && J_up >= J_down && dl >= 1 && L_min >= 0 &&
                     k_vec > 0.0,
                 "bad J range, DL, L_MIN or k");
  ChannelRanges ch;
  ch.n = n_channels;
  int s = 0;
  for (int c = 1; c <= n_channels; ++c) {  // channel c's states: [first[c-1], first[c])
    ch.first[c - 1] = s;
    while (s < n_states && indx_chann[s] == c) ++s;
  }
  ch.first[n_channels] = s;
  MQCT_ARG_CHECK(s == n_states,
                 "indx_chann must run over 1..n_channels in channel-major order (state %d)",
                 s + 1);
  if (mqct_device_count() <= 0) {
    set_error("no CUDA device available");
    return MQCT_E_NODEV;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int n_J = J_up - J_down + 1;
  channel_prob_kernel<<<(unsigned)n_traj, 128, 0, st>>>(d_amp, n_states, ch, d_prob);
  MQCT_CUDA_TRY(cudaGetLastError());
  const int64_t nt = (int64_t)n_J * n_channels;
  partial_sigma_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(
      d_prob, n_traj, n_channels, j_ini, J_down, n_J, L_min, dl, k_vec, d_partial);
  MQCT_CUDA_TRY(cudaGetLastError());
  sigma_kernel<<<(n_channels + 127) / 128, 128, 0, st>>>(d_partial, n_J, n_channels, d_sigma);
  MQCT_CUDA_TRY(cudaGetLastError());
  return MQCT_OK;
}
