// sa_runners.cu -- device-side drivers for single systems.
//
// sa_sys_anneal runs the reference's annealing<gpu_sys> loop
// (src/annealing.hpp:67-100) for one system on its stream without host
// round trips: `sweeps` sweeps per step, a measurement whenever i % stride == 0
// (i = sweep index inside the step), the running maximum of the float -H per
// replica (min_E), then the next temperature. The per-step temperatures,
// the draw base and the step index live in device memory, so one step is
// captured once as a CUDA graph and replayed for every step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "sa_b200.h"
#include "sa_device.cuh"
#include "sa_host.hpp"
#include "sa_measure.cuh"
#include "sa_system.hpp"

namespace sa {

struct AnnealState {
  unsigned long long draw_base;  // draw index of sweep 0 of the current step
  int step;                      // current step
  int pad;
  unsigned long long counts[128];
  double minE[64];               // running maximum of E + h*M (reference: min_E)
  int64_t lastE[64], lastM[64];
  int measured;
};

template <bool OPEN_X>
__global__ void __launch_bounds__(256) k_anneal_half_2d(word_t* __restrict__ s, const word_t* __restrict__ J,
                                                        int L, unsigned long long seed, const AnnealState* st,
                                                        int off, int c, const Thresholds* thr) {
  const Thresholds th = thr[st->step];
  const unsigned long long draw = st->draw_base + off;
  const int hL = L >> 1;
  const long half = (long)L * hL;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= half) return;
  const int r = (int)(t / hL), k = (int)(t - (long)r * hL);
  const int y = r, par = (c + y) & 1, x = 2 * k + par;
  int kw, ke;
  x_neighbours(k, par, hL, kw, ke);
  const int rn = wrap_dec(r, L), rs = wrap_inc(r, L);
  const word_t* so = s + (long)(1 - c) * half;
  word_t* sc = s + (long)c * half;
  const long idx = (long)r * hL + k;
  const word_t si = sc[idx];
  word_t mw = J[(long)c * half + idx] ^ so[(long)r * hL + kw] ^ si;
  word_t me = J[(long)(1 - c) * half + (long)r * hL + ke] ^ so[(long)r * hL + ke] ^ si;
  const word_t mn = J[(long)(2 + c) * half + idx] ^ so[(long)rn * hL + k] ^ si;
  const word_t ms = J[(long)(3 - c) * half + (long)rs * hL + k] ^ so[(long)rs * hL + k] ^ si;
  bool border = false;
  if (OPEN_X) {
    if (x == 0) { mw = ~0ULL; border = true; }
    if (x == L - 1) { me = ~0ULL; border = true; }
  }
  const uint32_t u = philox_draw(seed, (unsigned long long)x + (unsigned long long)L * y, draw);
  word_t c0, c1, c2;
  count4(mw, me, mn, ms, c0, c1, c2);
  uint32_t tdn, tup;
  if (OPEN_X && border) {
    tdn = prefix_count<4>(u, th.bdn);
    tup = prefix_count<4>(u, th.bup);
  } else {
    tdn = prefix_count<4>(u, th.dn);
    tup = prefix_count<4>(u, th.up);
  }
  sc[idx] = flip_word(si, c0, c1, c2, tdn, tup);
}

__global__ void __launch_bounds__(128) k_anneal_half_3d(word_t* __restrict__ s, const word_t* __restrict__ J,
                                                        int L, unsigned long long seed, const AnnealState* st,
                                                        int off, int c, const Thresholds* thr) {
  const Thresholds th = thr[st->step];
  const unsigned long long draw = st->draw_base + off;
  const int hL = L >> 1;
  const long plane = (long)L * hL;
  const long half = plane * L;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const int y = (int)(t / hL), k = (int)(t - (long)y * hL);
  const int par = (c + y) & 1, x = 2 * k + par;
  int kw, ke;
  x_neighbours(k, par, hL, kw, ke);
  const int yn = wrap_dec(y, L), ys = wrap_inc(y, L);
  const word_t* so = s + (long)(1 - c) * half;
  word_t* sc = s + (long)c * half;
  const word_t* Jxc = J + (long)c * half;
  const word_t* Jxo = J + (long)(1 - c) * half;
  const word_t* Jyc = J + (long)(2 + c) * half;
  const word_t* Jyo = J + (long)(3 - c) * half;
  const word_t* Jzc = J + (long)(4 + c) * half;
  word_t prev = sc[((long)(y + L * (L - 1))) * hL + k];
  word_t first = 0;
  for (int z = 0; z < L; ++z) {
    const long r = y + (long)L * z;
    const long idx = r * hL + k;
    const long rd = y + (long)L * (z == L - 1 ? 0 : z + 1);
    const word_t si = sc[idx];
    const word_t sd = (z == L - 1) ? first : sc[rd * hL + k];
    const word_t mw = Jxc[idx] ^ so[r * hL + kw] ^ si;
    const word_t me = Jxo[r * hL + ke] ^ so[r * hL + ke] ^ si;
    const word_t mn = Jyc[idx] ^ so[(yn + (long)L * z) * hL + k] ^ si;
    const word_t ms = Jyo[(ys + (long)L * z) * hL + k] ^ so[(ys + (long)L * z) * hL + k] ^ si;
    const word_t mu = Jzc[idx] ^ prev ^ si;
    const word_t md = Jzc[rd * hL + k] ^ sd ^ si;
    const uint32_t u = philox_draw(seed, (unsigned long long)x + (unsigned long long)L * r, draw);
    word_t c0, c1, c2;
    count6(mw, me, mn, ms, mu, md, c0, c1, c2);
    const word_t ns = flip_word(si, c0, c1, c2, prefix_count<6>(u, th.dn), prefix_count<6>(u, th.up));
    sc[idx] = ns;
    if (z == 0) first = ns;
    prev = ns;
  }
}

__global__ void __launch_bounds__(kMeasureThreads) k_anneal_measure(const word_t* __restrict__ s,
                                                                    const word_t* __restrict__ J, int L, int lattice,
                                                                    AnnealState* st) {
  __shared__ unsigned int sm[128];
  measure_block_counts(s, J, L, lattice, sm);
  for (int i = threadIdx.x; i < 128; i += blockDim.x)
    if (sm[i]) atomicAdd(&st->counts[i], (unsigned long long)sm[i]);
}

// E, M from the counts; -H = E + h*M as the reference's float; running max.
__global__ void k_anneal_fold(AnnealState* st, long nbonds, long N, double h) {
  const int j = threadIdx.x;
  if (j < 64) {
    const int64_t E = 2 * (int64_t)st->counts[j] - nbonds;
    const int64_t M = 2 * (int64_t)st->counts[64 + j] - N;
    const float v = (float)((double)E + h * (double)M);
    st->lastE[j] = E;
    st->lastM[j] = M;
    st->minE[j] = (st->measured == 0) ? (double)v : fmax(st->minE[j], (double)v);
  }
  __syncthreads();
  if (j < 128) st->counts[j] = 0;
  if (j == 0) st->measured += 1;
}

// end of a step: record its last energies, advance the step and the draw base
__global__ void k_anneal_step_end(AnnealState* st, int64_t* stepE, int sweeps) {
  const int j = threadIdx.x;
  if (j < 64 && stepE) stepE[(long)st->step * 64 + j] = st->lastE[j];
  __syncthreads();
  if (j == 0) {
    st->step += 1;
    st->draw_base += 2ULL * sweeps;
  }
}

}  // namespace sa

using namespace sa;

extern "C" int sa_sys_anneal(sa_system_t sy, const double* T, int nsteps, int sweeps, int stride, float* min_E,
                             int64_t* step_E) {
  if (!sy || !T || !min_E) return fail(SA_ERR_INVALID, "null argument");
  if (nsteps < 1 || sweeps < 1 || stride < 0) return fail(SA_ERR_INVALID, "bad schedule");
  std::vector<Thresholds> thr(nsteps);
  for (int k = 0; k < nsteps; ++k) {
    if (!(T[k] > 0)) return fail(SA_ERR_INVALID, "temperatures must be > 0");
    if (!make_thresholds(sy->lattice, T[k], sy->h, &thr[k])) return fail(SA_ERR_INVALID, "non-monotone table");
  }
  if (sy->rng_mode == SA_RNG_MT19937_64 || sy->first_colour != 0 || sy->split) {
    // the CPU reference's stream, or a system whose sweeps start with colour
    // 1: annealing<>'s own loop (src/annealing.hpp:67-100) over sa_sys_sweep /
    // sa_sys_measure
    std::vector<double> mn(64, 0.0);
    std::vector<int64_t> last(64, 0);
    int measured = 0;
    for (int k = 0; k < nsteps; ++k) {
      int st = sa_sys_set_T(sy, T[k]);
      for (int i = 0; st == SA_OK && i < sweeps; ++i) {
        st = sa_sys_sweep(sy, 1);
        if (st == SA_OK && stride != 0 && i % stride == 0) {
          int64_t E[64], M[64];
          st = sa_sys_measure(sy, E, M);
          for (int j = 0; st == SA_OK && j < 64; ++j) {
            const double v = (double)(float)((double)E[j] + sy->h * (double)M[j]);
            mn[j] = measured ? std::max(mn[j], v) : v;
            last[j] = E[j];
          }
          if (st == SA_OK) ++measured;
        }
      }
      if (st != SA_OK) return st;
      if (step_E) memcpy(step_E + (long)k * 64, last.data(), 64 * sizeof(int64_t));
    }
    for (int j = 0; j < 64; ++j) min_E[j] = measured ? (float)mn[j] : 0.f;
    sy->thr = thr[nsteps - 1];
    return SA_OK;
  }
  if (resident_ok(sy)) {
    // zero field: the whole schedule in one launch of the resident kernel
    int64_t emax[64];
    int measured = 0;
    const int st = resident_run(sy, T, nsteps, sweeps, stride, emax, step_E, &measured);
    if (st != SA_OK) return st;
    for (int j = 0; j < 64; ++j) min_E[j] = measured ? (float)emax[j] : 0.f;
    sy->T = T[nsteps - 1];
    sy->thr = thr[nsteps - 1];
    return SA_OK;
  }
  Thresholds* d_thr = nullptr;
  AnnealState* d_st = nullptr;
  int64_t* d_stepE = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int status = SA_OK;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_thr);
    cudaFree(d_st);
    cudaFree(d_stepE);
  };
#define SA_RUN_TRY(expr)                         \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) {                     \
      status = cuda_fail(e_, #expr);             \
      cleanup();                                 \
      return status;                             \
    }                                            \
  } while (0)
  SA_RUN_TRY(cudaMalloc(&d_thr, nsteps * sizeof(Thresholds)));
  SA_RUN_TRY(cudaMalloc(&d_st, sizeof(AnnealState)));
  if (step_E) SA_RUN_TRY(cudaMalloc(&d_stepE, (size_t)nsteps * 64 * sizeof(int64_t)));
  AnnealState h_st;
  memset(&h_st, 0, sizeof h_st);
  h_st.draw_base = sy->draw;
  SA_RUN_TRY(cudaMemcpyAsync(d_thr, thr.data(), nsteps * sizeof(Thresholds), cudaMemcpyHostToDevice, sy->stream));
  SA_RUN_TRY(cudaMemcpyAsync(d_st, &h_st, sizeof h_st, cudaMemcpyHostToDevice, sy->stream));
  SA_RUN_TRY(cudaStreamSynchronize(sy->stream));
  // one step as a graph
  const long per_block = (long)kMeasureThreads * kMeasureMaxSitesPerThread;
  long nb = (sy->N + kMeasureThreads * 8 - 1) / (kMeasureThreads * 8);
  if (nb > 1184) nb = 1184;
  nb = std::max(nb, (sy->N + per_block - 1) / per_block);
  if (nb < 1) nb = 1;
  SA_RUN_TRY(cudaStreamBeginCapture(sy->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < sweeps; ++i) {
    for (int c = 0; c < 2; ++c) {
      if (sy->lattice == SA_LATTICE_3D) {
        const long plane = (long)sy->L * (sy->L / 2);
        k_anneal_half_3d<<<(unsigned)((plane + 127) / 128), 128, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L, sy->seed,
                                                                                  d_st, 2 * i + c, c, d_thr);
      } else if (sy->lattice == SA_LATTICE_2D_OPEN_X) {
        k_anneal_half_2d<true><<<(unsigned)((sy->half + 255) / 256), 256, 0, sy->stream>>>(
            sy->d_s, sy->d_J, sy->L, sy->seed, d_st, 2 * i + c, c, d_thr);
      } else {
        k_anneal_half_2d<false><<<(unsigned)((sy->half + 255) / 256), 256, 0, sy->stream>>>(
            sy->d_s, sy->d_J, sy->L, sy->seed, d_st, 2 * i + c, c, d_thr);
      }
    }
    if (stride != 0 && i % stride == 0) {
      k_anneal_measure<<<(unsigned)nb, kMeasureThreads, 0, sy->stream>>>(sy->d_s, sy->d_J, sy->L, sy->lattice, d_st);
      k_anneal_fold<<<1, 128, 0, sy->stream>>>(d_st, sy->nbonds, sy->N, sy->h);
    }
  }
  k_anneal_step_end<<<1, 64, 0, sy->stream>>>(d_st, d_stepE, sweeps);
  cudaError_t ce = cudaStreamEndCapture(sy->stream, &graph);
  if (ce != cudaSuccess) {
    status = cuda_fail(ce, "cudaStreamEndCapture");
    cleanup();
    return status;
  }
  SA_RUN_TRY(cudaGraphInstantiate(&exec, graph, 0));
  for (int k = 0; k < nsteps; ++k) SA_RUN_TRY(cudaGraphLaunch(exec, sy->stream));
  SA_RUN_TRY(cudaMemcpyAsync(&h_st, d_st, sizeof h_st, cudaMemcpyDeviceToHost, sy->stream));
  if (step_E)
    SA_RUN_TRY(cudaMemcpyAsync(step_E, d_stepE, (size_t)nsteps * 64 * sizeof(int64_t), cudaMemcpyDeviceToHost,
                               sy->stream));
  SA_RUN_TRY(cudaStreamSynchronize(sy->stream));
  for (int j = 0; j < 64; ++j) min_E[j] = h_st.measured ? (float)h_st.minE[j] : 0.f;
  sy->draw += 2ULL * sweeps * nsteps;
  sy->T = T[nsteps - 1];
  sy->thr = thr[nsteps - 1];
  cleanup();
#undef SA_RUN_TRY
  return SA_OK;
}
