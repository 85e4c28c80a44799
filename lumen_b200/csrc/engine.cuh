// The engine's kernels and their launchers, shared by the library's translation units (lumen_b200.cu: the host side
// and the C ABI; k_part.cu: one part of the kernel instantiations each, compiled in parallel). A kernel template is
// instantiated in one part only: lumen_b200.cu declares every launcher it calls extern (LUMEN_SHAPES).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lumen_b200.h"
#include "dstep.cuh"

using namespace lb;

// ------------------------------------------------------------------------------------------- error handling
// the calling thread's last error message, and the kernels its last call launched (defined in lumen_b200.cu)
std::string& lumen_err();
long long& lumen_launches();
inline int set_err(int code, const std::string& m) {
  lumen_err() = m;
  return code;
}
#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return set_err(LUMEN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct LumenScene {
  DScene S;
  int dev;
  float* pool_live;
  float* pool_ref;  // == pool_live unless a distinct reference is set
  int n_pool;
  std::vector<void*> allocs;
  std::vector<int32_t> sigma_tabs;  // the sigma_alpha tables of the unified facet rows
  std::vector<int32_t> tab;         // host copy of the (offset, knots) table index
  std::vector<int32_t> spectrum_tabs;  // the WLS emission spectra's tables
  std::vector<std::pair<int, int>> roles;  // (table, admissible range) of every table a run reads
  int has_torus;                       // a leaf of typ 2: the launches run the kernels with the torus code
  int single;                          // every solid one quadric / plane leaf: the single-leaf instantiation
  int clip;                            // the extended locate is needed: a protrusion clip or frame groups
  int groups;                          // frame groups (the instantiation walking them)
  int nav64;                           // LUMEN_PREC_FLOAT64: S's vol_f, node_f, leaf_f, plane_f hold float64 data
  const float* vol_f32;                // the float32 frames (the readout groups' binning reads them in either precision)
  // the wavefront's rounds per photon a slot carries, from the last synchronous wavefront call (an estimate for the
  // asynchronous calls' fixed rounds; concurrent calls may overwrite one another's)
  mutable float wave_rpp = 0.0f;
};

// the position's precision of an instantiation: NAV64 = 1 the float64 navigator's (LUMEN_PREC_FLOAT64)
template <int NAV64> struct NavOf { using F = float; };
template <> struct NavOf<1> { using F = double; };

// --------------------------------------------------------------------------------------------- the kernels
struct Tally {
  int E, S_, nb, P;
  float bin0, bin_w;
  double *arrival, *arrival_t, *arrival2, *hist, *jac, *health;
  unsigned long long* counts;
  const double* cot;  // the adjoint's cotangent (E * S_) or null
  double* grads;      // the adjoint's output (P) or null
  unsigned long long* mt_key;  // the moment table: keys (photon << 32 | event x sensor cell), MT_EMPTY when free
  double* mt_sum;              // the photon's sum on that cell
  unsigned mt_mask;            // slots - 1 (a power of two)
};

// The moment table. The second moment (run.py:483 _moment_adds) squares each photon's own sum per cell; a photon keeps
// its first four sums in registers (PhotonTally) and the rest here: one slot per (photon, cell), claimed by a CAS and
// then written only by the photon's own thread (its sum is the sequential sum of its deposits, as in registers).
// k_moment_flush squares every slot into arrival2 and frees it after the launch. A slot is found within MT_PROBES
// linear probes or the sum is lost (squared alone, counts[LUMEN_C_MOMENT_LOST]). mt_add returns 1 where it claimed
// a slot (the photon's first deposit on that cell past its first four sensors), 2 where it added to the photon's own
// slot, 0 where the table had no room.
#define MT_EMPTY 0xffffffffffffffffull
#define MT_PROBES 64

__device__ __forceinline__ int mt_add(const Tally& T, unsigned pid, unsigned cell, double v) {
  const unsigned long long k = ((unsigned long long)pid << 32) | cell;
  unsigned h = (unsigned)((k * 0x9E3779B97F4A7C15ull) >> 32) & T.mt_mask;
  for (int p = 0; p < MT_PROBES; ++p) {
    unsigned long long old = T.mt_key[h];  // a key once written stays for the launch: a non-empty read is final
    if (old == MT_EMPTY) old = atomicCAS(T.mt_key + h, MT_EMPTY, k);
    if (old == MT_EMPTY) { T.mt_sum[h] = v; return 1; }
    if (old == k) { T.mt_sum[h] += v; return 2; }
    h = (h + 1) & T.mt_mask;
  }
  return 0;
}

struct Launch {
  Run R;
  LumenRows rows;
  LumenSource src;
  int use_rows;
  Key key;
  int64_t first_id, n;
  unsigned long long* next;  // the photon counter
  int* abort_flag;
  long long step_budget;
  unsigned long long* steps_used;
  int budget_chunk;  // steps a thread of the persistent loop counts before it adds them to steps_used (1 .. 256)
  Tally T;
  float* truth;  // the photons' analog records (truth rows, LUMEN_F_TRUTH: the ANALOG instantiation), else null
  // the wavefront's slots a persistent launch resumes before it takes new photons (its drain: one thread a slot), or
  // wv_W = 0
  const uint32_t* wv_ph;
  const uint32_t* wv_ex;
  const float* wv_dw;
  const int32_t* wv_act;
  int wv_W;
  const int32_t* ev_vol;  // per event its start volume (point-like sources: k_event_locate), or null
};

// what picks a launch's instantiation, host side: the scene has a torus leaf; the run keeps truth rows
struct Pick {
  int torus;
  int single;              // every solid a single quadric / plane leaf
  int clip;                // a protrusion clip (the wavefront's fill locates without the extended rule)
  int groups;              // frame groups: the extended instantiation with their traversal
  int analog;
  int nav64;               // the scene's navigator is float64
  int born;                // a sensor counts the photons born inside it (the wavefront's step kernel with that branch)
  const float* vol_f32;    // the scene's float32 frames (the readout binning)
};

#define CACHE 4

// the current photon's first four per-sensor sums (the second moment squares each at the photon's end); read and
// written by constant index only, so they stay in registers; pid is the photon's index in the call (the moment
// table's key for its further sums)
struct PhotonTally {
  int sensor[CACHE];
  double sum[CACHE];
  int n;
  unsigned pid;
};

__device__ __forceinline__ void flush2(const Tally& T, int e, int s, double v) {
  if ((unsigned)e >= (unsigned)T.E || (unsigned)s >= (unsigned)T.S_) return;
  if (T.arrival2) atomicAdd(T.arrival2 + (size_t)e * T.S_ + s, v * v);
}

__device__ __forceinline__ void flush_all(const Tally& T, int e, PhotonTally& pt) {
#pragma unroll
  for (int j = 0; j < CACHE; ++j)
    if (j < pt.n) flush2(T, e, pt.sensor[j], pt.sum[j]);
}

// adds every lane's non-zero health fates (times its row weight) to the block's shared sums: a warp sum first, then
// one shared atomic per fate and warp (lanes with nothing to add pass zeros; every lane of the warp must call it)
__device__ __forceinline__ void health_add(double* sh, const Dep& dep, double w0, int on) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    float f = on ? (k < 8 ? dep.fates[k] : dep.pushed) : 0.0f;
    if (!__any_sync(FULL, f != 0.0f)) continue;
    double v = f != 0.0f ? (double)f * w0 : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if (lane == 0) atomicAdd(sh + (k < 8 ? k : LUMEN_H_PUSHED), v);
  }
}

// adds v (per lane, 0 for none) to a shared sum: one warp sum and one atomic per warp (every lane must call it)
__device__ __forceinline__ void warp_add(double* sh, double v) {
  const unsigned FULL = 0xffffffffu;
  if (!__any_sync(FULL, v != 0.0)) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sh, v);
}

// adds one deposit to the tallies; returns 0, or 1 where it opened a sum in the moment table (a sensor past the
// photon's first four), or 2 where the table had no room (the deposit squared alone)
template <int G>
__device__ __forceinline__ int deposit(const Tally& T, int e, const Dep& dep, const float* dq, double w0,
                                       PhotonTally& pt) {
  int s = dep.sensor;
  if ((unsigned)e >= (unsigned)T.E || (unsigned)s >= (unsigned)T.S_) return 0;  // an event or sensor out of range
  double v = (double)dep.q * w0;
  size_t ix = (size_t)e * T.S_ + s;
  if (T.arrival) {
    atomicAdd(T.arrival + ix, v);
    atomicAdd(T.arrival_t + ix, v * (double)dep.time);
  }
  if (T.nb > 0) {
    float b = floorf((dep.time - T.bin0) / T.bin_w);
    if (b >= 0.0f && b < (float)T.nb) atomicAdd(T.hist + ix * T.nb + (size_t)b, v);
  }
  if (G > 0) {
    if (T.jac)
      for (int p = 0; p < T.P; ++p) atomicAdd(T.jac + ix * T.P + p, (double)dq[p] * w0);
    if (T.cot) {
      double c = T.cot[ix];
      if (c != 0.0)
        for (int p = 0; p < T.P; ++p) atomicAdd(T.grads + p, c * (double)dq[p] * w0);
    }
  }
  if (v == 0.0 || !T.arrival2) return 0;  // a deposit of 0 (a photon of weight 0) adds nothing to any sum
  int found = 0;
#pragma unroll
  for (int j = 0; j < CACHE; ++j)
    if (j < pt.n && pt.sensor[j] == s) { pt.sum[j] += v; found = 1; }
  if (found) return 0;
  if (pt.n < CACHE) {
#pragma unroll
    for (int j = 0; j < CACHE; ++j)
      if (j == pt.n) { pt.sensor[j] = s; pt.sum[j] = v; }
    pt.n += 1;
    return 0;
  }
  const int m = T.mt_key ? mt_add(T, pt.pid, (unsigned)ix, v) : 0;
  if (m) return m == 1;
  atomicAdd(T.arrival2 + ix, v * v);
  return 2;
}

__device__ __forceinline__ void get_row(const Launch& L, int64_t i, Row& r) {
  if (L.use_rows) d_rows_row(L.rows, i, r);
  else d_source_row(L.R.S, L.R.live, L.R.ref, L.src, L.key, L.first_id + i, r);
  r.vol = L.ev_vol ? __ldg(L.ev_vol + r.event) : -1;
}

// every point-like event's start volume, located once per call (Launch.ev_vol: the point and time sources, whose
// photons all start at the event's point; the same locate as each photon's would be, EXT the run's)
template <int EXT>
__global__ void k_event_locate(DScene S, LumenSource src, int32_t* ev_vol) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= src.n_events) return;
  const float* f = src.ev_f + (size_t)e * LUMEN_EV_F;
  float x[3] = {__ldg(f), __ldg(f + 1), __ldg(f + 2)};
  ev_vol[e] = nav_locate<EXT>(S, x);
}

struct WaveExtra {  // what a slot carries besides the photon: its key, event, row weight and sensor-sum cache
  Key pkey;
  int ev, pad;
  double w0;
  PhotonTally pt;
};

struct Wave {
  uint32_t* ph;     // W x sizeof(Photon) / 4
  uint32_t* ex;     // W x sizeof(WaveExtra) / 4
  uint32_t* pre;    // W x sizeof(Pre) / 4
  uint32_t* q;      // W x sizeof(Query) / 4
  float* dw;        // W x LUMEN_MAX_GRAD (gradient runs)
  int32_t* act;     // W: the slot holds a live photon
  unsigned long long* live;  // slots live after the last k_wave_step (zeroed before each)
  int W;
};

template <class T>
__device__ __forceinline__ void wv_ld(const uint32_t* b, int W, int i, T& v) {
  static_assert(sizeof(T) % 4 == 0, "word-major records hold whole words");
  uint32_t* w = reinterpret_cast<uint32_t*>(&v);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(T) / 4); ++k) w[k] = b[(size_t)k * W + i];
}
template <class T>
__device__ __forceinline__ void wv_st(uint32_t* b, int W, int i, const T& v) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(&v);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(T) / 4); ++k) b[(size_t)k * W + i] = w[k];
}

// The persistent photon loop: a lane refill per step (src/lumen/run.py:81 SCHEDULE = "step").
// Launch shapes (LumenControls.variant): 0 = 256 threads x 4 blocks per SM (64 registers, 32 warps an SM: the
// measured best of 128 / 256 threads at 1-8 blocks on the tank: the loop is latency- and divergence-bound, so warps
// to switch between beat registers), 1 = 128 x 8 (64 registers), 2 = 256 x 3 (85 registers). The autotuner
// (lumen_b200/autotune.py) picks one per workload. TORUS: the extended-geometry instantiation (torus
// leaves and mesh chunks), run for scenes with either (shape 0 only); the others are compiled without that code, so a
// scene of quadric and plane leaves pays nothing for it.
// ANALOG: each photon carries its analog photon and writes its record (truth rows: LUMEN_F_TRUTH; G = 0, shape 0).
// NAV64: the float64 navigator and position (a LUMEN_PREC_FLOAT64 scene; shape 0, with the torus code).
template <int G, int BLOCK, int MINB, int TORUS, int ANALOG = 0, int NAV64 = 0>
__global__ void __launch_bounds__(BLOCK, MINB) k_trace(Launch L) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  PhotonT<typename NavOf<NAV64>::F> ph;
  float dw[G > 0 ? G : 1], dq[G > 0 ? G : 1];
  PhotonTally pt;
  pt.n = 0;
  Key pkey = {0u, 0u};
  int active = 0, ev = 0;
  double w0 = 0.0;
  Ana an;
  int64_t gi = 0;
  // the health fates, summed per block in shared memory (a step adds its non-zero fates times the row weight): no
  // per-thread accumulators stay live across the step
  __shared__ double sh_health[LUMEN_N_HEALTH];
  if (threadIdx.x < LUMEN_N_HEALTH) sh_health[threadIdx.x] = 0.0;
  __syncthreads();
  unsigned c_ph = 0, c_steps = 0, c_dep = 0, c_trunc = 0, c_multi = 0, c_lost = 0;
  int budget_chunk = 0;
  if constexpr (!ANALOG && !NAV64) {
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    if (i < L.wv_W && L.wv_act[i]) {  // a wavefront slot's photon, where its last round left it
      WaveExtra ex;
      wv_ld(L.wv_ph, L.wv_W, i, ph);
      wv_ld(L.wv_ex, L.wv_W, i, ex);
      pkey = ex.pkey;
      ev = ex.ev;
      w0 = ex.w0;
      pt = ex.pt;
      if (G > 0)
        for (int p = 0; p < L.R.P; ++p) dw[p] = L.wv_dw[(size_t)p * L.wv_W + i];
      active = 1;
    }
  }
  for (;;) {
    unsigned need = __ballot_sync(FULL, !active);
    if (need) {
      int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      int abort_now = 0;
      if (lane == leader) {
        abort_now = L.abort_flag && *(volatile int*)L.abort_flag;
        base = abort_now ? (unsigned long long)L.n : atomicAdd(L.next, (unsigned long long)__popc(need));
      }
      base = __shfl_sync(FULL, base, leader);
      if (!active) {
        unsigned long long g = base + __popc(need & ((1u << lane) - 1u));
        if (g < (unsigned long long)L.n) {
          Row r;
          get_row(L, (int64_t)g, r);
          d_start<(TORUS & 1)>(L.R.S, r, ph);
          pkey = fold_in(L.key, (uint32_t)(L.first_id + (int64_t)g));
          w0 = (double)r.w0;
          ev = r.event;
          active = 1;
          pt.n = 0;
          pt.pid = (unsigned)g;
          if (G > 0)
            for (int p = 0; p < L.R.P; ++p) dw[p] = 0.0f;
          if (ANALOG) {  // run.py:319: one uniform of its own stream, open with probability k (state.py:58)
            float u = uniform(fold_in(pkey, D_ANALOG_STREAM), 0);
            an.k = r.w0;
            an.x = u < an.k ? u / (an.k > 0.0f ? an.k : 1.0f) : __int_as_float(0x7f800000);
            an.sensor = -1;
            an.time = 0.0f; an.lam = 0.0f; an.scale = 1.0f;
            an.pos[0] = an.pos[1] = an.pos[2] = 0.0f;
            an.vol = -1;
            gi = (int64_t)g;
          }
        }
      }
    }
    if (__ballot_sync(FULL, active) == 0) break;
    Dep dep;
    int stepped = active;
    double start_w = 0.0, trunc_w = 0.0;
    if (active) d_step<G, TORUS, ANALOG>(L.R, ph, dw, pkey, dep, dq, an);
    health_add(sh_health, dep, w0, stepped);
    if (active) {
      c_steps++;
      if (dep.sensor >= 0) {
        const int m = deposit<G>(L.T, ev, dep, dq, w0, pt);
        c_multi += m == 1;
        c_lost += m == 2;
        c_dep++;
      }
      if (!ph.alive || ph.vertex >= L.R.max_vertices) {
        flush_all(L.T, ev, pt);
        if (L.R.rec && ph.last >= 0) d_record_head(L.R, ph.last, (float)w0, ev);
        if (ANALOG) {  // the photon's analog record (run.py:350 per_item)
          float* tr = L.truth + (size_t)gi * LUMEN_TRUTH_WORDS;
          tr[LUMEN_TR_SENSOR] = __int_as_float(an.sensor);
          tr[LUMEN_TR_TIME] = an.time;
          tr[LUMEN_TR_LAM] = an.lam;
          tr[LUMEN_TR_SCALE] = an.scale;
          tr[LUMEN_TR_POS] = an.pos[0]; tr[LUMEN_TR_POS + 1] = an.pos[1]; tr[LUMEN_TR_POS + 2] = an.pos[2];
          tr[LUMEN_TR_VOL] = __int_as_float(an.vol);
        }
        if (ph.alive) {
          trunc_w = (double)ph.w * w0;
          c_trunc++;
        }
        start_w = w0;
        c_ph++;
        active = 0;
      }
      if (L.step_budget > 0 && ++budget_chunk == L.budget_chunk) {
        unsigned long long used = atomicAdd(L.steps_used, (unsigned long long)budget_chunk) + budget_chunk;
        // the first thread past the budget raises the flag and counts the abort, once per call
        if (used > (unsigned long long)L.step_budget && atomicExch(L.abort_flag, 1) == 0)
          atomicAdd(L.T.counts + LUMEN_C_ABORTED, 1ull);
        budget_chunk = 0;
      }
      if (L.abort_flag && *(volatile int*)L.abort_flag) active = 0;
    }
    warp_add(sh_health + LUMEN_H_START, start_w);
    warp_add(sh_health + LUMEN_H_TRUNCATED, trunc_w);
  }
  // the block's health and counters: one atomic per block and value
  __shared__ unsigned long long sc[LUMEN_N_COUNT][BLOCK / 32];
  const int warp = threadIdx.x >> 5;
  unsigned long long cv[LUMEN_N_COUNT] = {};
  cv[LUMEN_C_PHOTONS] = c_ph;
  cv[LUMEN_C_STEPS] = c_steps;
  cv[LUMEN_C_DEPOSITS] = c_dep;
  cv[LUMEN_C_TRUNCATED] = c_trunc;
  cv[LUMEN_C_MULTI] = c_multi;
  cv[LUMEN_C_MOMENT_LOST] = c_lost;
#pragma unroll
  for (int k = 0; k < LUMEN_N_COUNT; ++k) {
    unsigned long long v = cv[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    if (lane == 0) sc[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < LUMEN_N_HEALTH) {
    double v = sh_health[threadIdx.x];
    if (v != 0.0) atomicAdd(L.T.health + threadIdx.x, v);
  } else if (threadIdx.x >= 32 && threadIdx.x < 32 + LUMEN_N_COUNT) {
    int k = threadIdx.x - 32;
    unsigned long long v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sc[k][w];
    if (v) atomicAdd(L.T.counts + k, v);
  }
}

// ------------------------------------------------------------------------------------------------ the wavefront
// The photon loop as rounds over a pool of W slots held in HBM (launch variant LUMEN_VARIANT_WAVEFRONT): per round,
// k_wave_query runs every live slot's step up to and including its navigator query, and k_wave_step the rest of the
// step, the deposit, the photon's end and the slot's refill from the source. Each kernel is a part of the
// megakernel's code with its own registers; the state crosses HBM between them, word-major (word k of slot i at
// buf[k * W + i]) so that every load and store of a warp is one contiguous 128-byte access.
template <int G, int TORUS>
__global__ void __launch_bounds__(256, 3) k_wave_query(Launch L, Wave V) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.W || !V.act[i]) return;
  if (L.abort_flag && *(volatile int*)L.abort_flag) return;
  Photon ph;
  WaveExtra ex;
  wv_ld(V.ph, V.W, i, ph);
  wv_ld(V.ex, V.W, i, ex);
  Pre pr;
  d_pre<(TORUS & 1)>(L.R, ph, ex.pkey, pr);
  Query q = d_step_query<TORUS>(L.R, ph, pr);
  wv_st(V.ph, V.W, i, ph);
  wv_st(V.pre, V.W, i, pr);
  wv_st(V.q, V.W, i, q);
}

// BORN: the scene has a sensor that counts the photons born inside it (the branch of their first step, which reads
// none of the query the query kernel made for it; a scene without one runs the kernel compiled without the branch,
// the branch costs the tank's plain forward 2 % where it is compiled in)
template <int G, int BORN>
__global__ void __launch_bounds__(256, 2) k_wave_step(Launch L, Wave V) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  __shared__ double sh_health[LUMEN_N_HEALTH];
  __shared__ unsigned long long sc[LUMEN_N_COUNT + 1][8];
  if (threadIdx.x < LUMEN_N_HEALTH) sh_health[threadIdx.x] = 0.0;
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int in = i < V.W;
  int aborted = L.abort_flag && *(volatile int*)L.abort_flag;
  int act = in && !aborted && V.act[i];
  unsigned c_ph = 0, c_steps = 0, c_dep = 0, c_trunc = 0, c_multi = 0, c_lost = 0;
  Photon ph;
  WaveExtra ex;
  float dw[G > 0 ? G : 1], dq[G > 0 ? G : 1];
  Dep dep;
  const int stepped = act;
  double start_w = 0.0, trunc_w = 0.0;
  if (act) {
    wv_ld(V.ph, V.W, i, ph);
    wv_ld(V.ex, V.W, i, ex);
    if (G > 0)
      for (int p = 0; p < L.R.P; ++p) dw[p] = V.dw[(size_t)p * V.W + i];
    Ana an;
    const int bp = BORN ? d_born_entry(L.R.S, ph) : -2;
    if (bp != -2) {
      d_born<G>(L.R, ph, dw, bp, dep, dq, an);
    } else {
      Pre pr;
      Query q;
      wv_ld(V.pre, V.W, i, pr);
      wv_ld(V.q, V.W, i, q);
      d_post<G>(L.R, ph, dw, pr, q, dep, dq, an);
    }
    c_steps++;
    if (dep.sensor >= 0) {
      const int m = deposit<G>(L.T, ex.ev, dep, dq, ex.w0, ex.pt);
      c_multi += m == 1;
      c_lost += m == 2;
      c_dep++;
    }
    if (!ph.alive || ph.vertex >= L.R.max_vertices) {
      flush_all(L.T, ex.ev, ex.pt);
      if (L.R.rec && ph.last >= 0) d_record_head(L.R, ph.last, (float)ex.w0, ex.ev);
      if (ph.alive) {
        trunc_w = (double)ph.w * ex.w0;
        c_trunc++;
      }
      start_w = ex.w0;
      c_ph++;
      act = 0;
    }
  }
  health_add(sh_health, dep, stepped ? ex.w0 : 0.0, stepped);
  warp_add(sh_health + LUMEN_H_START, start_w);
  warp_add(sh_health + LUMEN_H_TRUNCATED, trunc_w);
  // the refill: free slots take consecutive photon ids, one atomic per warp
  int need = in && !act && !aborted;
  unsigned m = __ballot_sync(FULL, need);
  if (m) {
    int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(L.next, (unsigned long long)__popc(m));
    base = __shfl_sync(FULL, base, leader);
    if (need) {
      unsigned long long g = base + __popc(m & ((1u << lane) - 1u));
      if (g < (unsigned long long)L.n) {
        Row r;
        get_row(L, (int64_t)g, r);
        d_start(L.R.S, r, ph);
        ex.pkey = fold_in(L.key, (uint32_t)(L.first_id + (int64_t)g));
        ex.w0 = (double)r.w0;
        ex.ev = r.event;
        ex.pad = 0;
        ex.pt.n = 0;
        ex.pt.pid = (unsigned)g;
        if (G > 0)
          for (int p = 0; p < L.R.P; ++p) dw[p] = 0.0f;
        act = 1;
      }
    }
  }
  if (in) {
    if (act) {
      wv_st(V.ph, V.W, i, ph);
      wv_st(V.ex, V.W, i, ex);
      if (G > 0)
        for (int p = 0; p < L.R.P; ++p) V.dw[(size_t)p * V.W + i] = dw[p];
    }
    V.act[i] = act;
  }
  // the block's health, counters and live slots: one atomic per block and value
  const int warp = threadIdx.x >> 5;
  unsigned long long cv[LUMEN_N_COUNT + 1] = {};
  cv[LUMEN_C_PHOTONS] = c_ph;
  cv[LUMEN_C_STEPS] = c_steps;
  cv[LUMEN_C_DEPOSITS] = c_dep;
  cv[LUMEN_C_TRUNCATED] = c_trunc;
  cv[LUMEN_C_MULTI] = c_multi;
  cv[LUMEN_C_MOMENT_LOST] = c_lost;
  cv[LUMEN_N_COUNT] = (unsigned long long)act;  // the live slots
#pragma unroll
  for (int k = 0; k < LUMEN_N_COUNT + 1; ++k) {
    unsigned long long v = cv[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    if (lane == 0) sc[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < LUMEN_N_HEALTH) {
    double v = sh_health[threadIdx.x];
    if (v != 0.0) atomicAdd(L.T.health + threadIdx.x, v);
  } else if (threadIdx.x >= 32 && threadIdx.x < 32 + LUMEN_N_COUNT + 1) {
    int k = threadIdx.x - 32;
    unsigned long long v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sc[k][w];
    if (v) atomicAdd(k < LUMEN_N_COUNT ? L.T.counts + k : V.live, v);
    if (k == LUMEN_C_STEPS && v && L.step_budget > 0) {  // the call's step budget, counted per block
      unsigned long long used = atomicAdd(L.steps_used, v) + v;
      if (used > (unsigned long long)L.step_budget && atomicExch(L.abort_flag, 1) == 0)
        atomicAdd(L.T.counts + LUMEN_C_ABORTED, 1ull);
    }
  }
}

// One thread per photon to its end: the per-photon record the parity tests compare exactly.
template <int NAV64>
__global__ void k_trace_photons(Launch L, int32_t* out_i, float* out_f) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  Row r;
  get_row(L, i, r);
  PhotonT<typename NavOf<NAV64>::F> ph;
  d_start<1>(L.R.S, r, ph);
  Key pkey = fold_in(L.key, (uint32_t)(L.first_id + i));
  float dw[1], dq[1];
  int n_dep = 0, first_sensor = -1;
  double sum_q = 0.0, sum_qt = 0.0;
  while (ph.alive && ph.vertex < L.R.max_vertices) {
    Dep dep;
    Ana an;
    d_step<0, 3>(L.R, ph, dw, pkey, dep, dq, an);  // every geometry: tori, meshes, clips, frame groups
    if (dep.sensor >= 0) {
      n_dep++;
      if (first_sensor < 0) first_sensor = dep.sensor;
      sum_q += (double)dep.q;
      sum_qt += (double)dep.q * (double)dep.time;
    }
  }
  out_i[5 * i + 0] = ph.vertex;
  out_i[5 * i + 1] = n_dep;
  out_i[5 * i + 2] = ph.alive ? 0 : 1;
  out_i[5 * i + 3] = first_sensor;
  out_i[5 * i + 4] = ph.vol;
  out_f[4 * i + 0] = (float)sum_q;
  out_f[4 * i + 1] = ph.w;
  out_f[4 * i + 2] = ph.t;
  out_f[4 * i + 3] = (float)sum_qt;
}

template <class NF>
__global__ void k_query(DScene S, const NF* ray, const int32_t* vol, const int32_t* srf, NF t_max, int64_t n,
                        int32_t* out_i, NF* out_f) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  NF o[3] = {ray[6 * i], ray[6 * i + 1], ray[6 * i + 2]};
  NF d[3] = {ray[6 * i + 3], ray[6 * i + 4], ray[6 * i + 5]};
  int known = vol[i] >= 0 && vol[i] <= S.n;
  int v = known ? vol[i] : nav_locate<1>(S, o);
  int last = known ? srf[i] : -1;
  QueryT<NF> q = nav_query<3>(S, o, d, v, t_max, last, nullptr, sizeof(NF) == 4 ? (NF)D_HUGE : (NF)1e30);
  int32_t* oi = out_i + 8 * i;
  oi[0] = q.hit; oi[1] = q.vol_before; oi[2] = q.vol_after; oi[3] = q.cls_before; oi[4] = q.cls_after;
  oi[5] = q.srf; oi[6] = q.zero;
  oi[7] = q.hit ? vI(S, q.vol_after, LUMEN_VI_SENSOR) : -1;
  NF* of = out_f + 4 * i;
  of[0] = q.t; of[1] = q.normal[0]; of[2] = q.normal[1]; of[3] = q.normal[2];
}

template <class NF>
__global__ void k_locate(DScene S, const NF* pts, int64_t n, int32_t* vol) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  NF x[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  vol[i] = nav_locate<1>(S, x);
}

inline int grid_for(const void* fn, int block, int* grid) {
  int dev = 0, sms = 0, per = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0));
  *grid = sms * (per > 0 ? per : 1);
  return 0;
}

// blocks > 0: that grid instead of the resident one (the wavefront's drain: one thread a slot)
template <int G, int BLOCK, int MINB, int TORUS, int ANALOG = 0, int NAV64 = 0>
int launch_shape(const Launch& L, int bps, cudaStream_t stream, int blocks) {
  int grid = 0, st = 0;
  if (blocks > 0) grid = blocks;
  else if ((st = grid_for((const void*)k_trace<G, BLOCK, MINB, TORUS, ANALOG, NAV64>, BLOCK, &grid))) return st;
  if (bps > 0 && blocks <= 0) {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (sms * bps < grid) grid = sms * bps;
  }
  // a budget's steps are counted in chunks small enough that the grid's threads cannot overrun it by more than a
  // quarter, and at most 256 steps (one atomic per 256 steps of a thread)
  Launch LB = L;
  const long long per = L.step_budget / (4LL * grid * BLOCK);
  LB.budget_chunk = (int)(per < 1 ? 1 : (per > 256 ? 256 : per));
  k_trace<G, BLOCK, MINB, TORUS, ANALOG, NAV64><<<grid, BLOCK, 0, stream>>>(LB);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

// The wavefront's rounds (LUMEN_VARIANT_WAVEFRONT): a fill, then query and step kernels, then the drain: the
// persistent loop resumes every slot still live (one thread a slot) and takes the photons left. A synchronous call
// reads the live slots back every fourth round and drains once fewer than a 64th of the slots are live (the tail,
// where a round's launches cost more than its few steps: measured against an 8th, 16th, 32nd, 256th and 1024th); an asynchronous one (LUMEN_F_ASYNC) runs `rounds` rounds
// without a readback (<= 0: *rpp rounds per photon a slot carries, the scene's estimate from its last synchronous
// call) and drains. The pool holds up to LUMEN_WAVE_POOL slots (about 350 bytes each with gradients), allocated on the
// call's stream.
#define LUMEN_WAVE_POOL (1 << 21)
template <int G>
int run_wave(const Launch& L, const Pick& pk, unsigned long long* live, cudaStream_t stream, int slots_log2,
             int async, int rounds, float* rpp) {
  const int64_t pool = slots_log2 >= 16 && slots_log2 <= 23 ? (int64_t)1 << slots_log2 : (int64_t)LUMEN_WAVE_POOL;
  int64_t want = L.n < pool ? L.n : pool;
  int W = (int)((want + 255) / 256 * 256);
  const size_t nph = sizeof(Photon) / 4, nex = sizeof(WaveExtra) / 4, npre = sizeof(Pre) / 4, nq = sizeof(Query) / 4;
  const size_t ng = G > 0 ? LUMEN_MAX_GRAD : 0;
  size_t words = (size_t)W * (nph + nex + npre + nq + ng + 1);
  uint32_t* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, words * 4, stream));
  Wave V;
  V.W = W;
  V.ph = buf;
  V.ex = V.ph + (size_t)W * nph;
  V.pre = V.ex + (size_t)W * nex;
  V.q = V.pre + (size_t)W * npre;
  V.dw = (float*)(V.q + (size_t)W * nq);
  V.act = (int32_t*)(V.dw + (size_t)W * ng);
  V.live = live;
  const int grid = W / 256;
  CK(cudaMemsetAsync(V.act, 0, (size_t)W * 4, stream));
  if (pk.born) k_wave_step<G, 1><<<grid, 256, 0, stream>>>(L, V);  // the fill: every slot takes a photon
  else k_wave_step<G, 0><<<grid, 256, 0, stream>>>(L, V);
  CK(cudaGetLastError());
  ++lumen_launches();
  const long long per_slot = (L.n + W - 1) / W;  // photons a slot carries in turn
  long long cap = -1;                             // rounds of an asynchronous call
  if (async) {
    const float est = rpp && *rpp > 0.0f ? *rpp : 3.0f;
    cap = rounds > 0 ? rounds : (long long)ceilf(est * (float)per_slot);
  }
  long long r = 0;
  int drained = 0;
  for (;; ++r) {
    if (async && r >= cap) break;
    if (pk.torus) k_wave_query<G, 1><<<grid, 256, 0, stream>>>(L, V);
    else if (pk.single) k_wave_query<G, 2><<<grid, 256, 0, stream>>>(L, V);
    else k_wave_query<G, 0><<<grid, 256, 0, stream>>>(L, V);
    CK(cudaMemsetAsync(V.live, 0, sizeof(unsigned long long), stream));
    if (pk.born) k_wave_step<G, 1><<<grid, 256, 0, stream>>>(L, V);
    else k_wave_step<G, 0><<<grid, 256, 0, stream>>>(L, V);
    CK(cudaGetLastError());
    lumen_launches() += 2;
    if (!async && (r & 3) == 3) {
      unsigned long long h = 0;
      CK(cudaMemcpyAsync(&h, V.live, sizeof(h), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (h == 0) break;
      if (h < (unsigned long long)(W / 64)) {
        drained = 1;
        ++r;
        break;
      }
    }
  }
  if (async || drained) {  // the persistent loop finishes the live slots and takes the photons left
    Launch LD = L;
    LD.wv_ph = V.ph;
    LD.wv_ex = V.ex;
    LD.wv_dw = V.dw;
    LD.wv_act = V.act;
    LD.wv_W = W;
    int st = pk.torus ? launch_shape<G, 256, 4, 1>(LD, 0, stream, grid)
                      : (pk.single ? launch_shape<G, 256, 4, 2>(LD, 0, stream, grid)
                                   : launch_shape<G, 256, 4, 0>(LD, 0, stream, grid));  // fmt: skip
    if (st) return st;
  }
  if (!async && rpp && per_slot > 0) *rpp = (float)r / (float)per_slot;
  CK(cudaFreeAsync(buf, stream));
  return 0;
}

// the per-photon, query and locate kernels' launchers (one thread each)
template <int NAV64>
int launch_photons(const Launch& L, int32_t* out_i, float* out_f, cudaStream_t stream) {
  const int block = 128;
  const int64_t grid = (L.n + block - 1) / block;
  k_trace_photons<NAV64><<<(unsigned)grid, block, 0, stream>>>(L, out_i, out_f);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

template <class NF>
int launch_query(const DScene& S, const NF* ray, const int32_t* vol, const int32_t* srf, NF t_max, int64_t n,
                 int32_t* out_i, NF* out_f, cudaStream_t stream) {
  const int block = 128;
  k_query<<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(S, ray, vol, srf, t_max, n, out_i, out_f);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

template <class NF>
int launch_locate(const DScene& S, const NF* pts, int64_t n, int32_t* vol, cudaStream_t stream) {
  const int block = 128;
  k_locate<<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(S, pts, n, vol);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

template <int EXT>
int launch_event_locate(const DScene& S, const LumenSource& src, int32_t* ev_vol, cudaStream_t stream) {
  const int block = 128;
  k_event_locate<EXT><<<(unsigned)((src.n_events + block - 1) / block), block, 0, stream>>>(S, src, ev_vol);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

// Every k_trace instantiation a launch may pick (G, BLOCK, MINB, TORUS, ANALOG, NAV64), in the parts of the build
#define LUMEN_SHAPES_0(X) X(0, 256, 4, 2, 0, 0) X(0, 256, 3, 2, 0, 0) X(0, 128, 8, 2, 0, 0)
#define LUMEN_SHAPES_1(X) X(0, 256, 4, 0, 0, 0) X(0, 256, 3, 0, 0, 0) X(0, 128, 8, 0, 0, 0)
#define LUMEN_SHAPES_2(X) X(0, 256, 4, 1, 0, 0) X(0, 256, 4, 3, 0, 0)
#define LUMEN_SHAPES_3(X) X(0, 256, 4, 0, 1, 0) X(0, 256, 4, 1, 1, 0) X(0, 256, 4, 3, 1, 0)
#define LUMEN_SHAPES_4(X) X(8, 256, 4, 2, 0, 0) X(8, 256, 3, 2, 0, 0) X(8, 128, 8, 2, 0, 0)
#define LUMEN_SHAPES_5(X) X(8, 256, 4, 0, 0, 0) X(8, 256, 3, 0, 0, 0) X(8, 128, 8, 0, 0, 0)
#define LUMEN_SHAPES_6(X) X(8, 256, 4, 1, 0, 0) X(8, 256, 4, 3, 0, 0)
#define LUMEN_SHAPES_7(X) X(0, 256, 4, 1, 1, 1) X(0, 256, 4, 3, 1, 1) X(0, 256, 4, 2, 0, 1)
#define LUMEN_SHAPES_8(X) X(0, 256, 4, 3, 0, 1) X(0, 256, 4, 1, 0, 1)
#define LUMEN_SHAPES_9(X) X(8, 256, 4, 2, 0, 1) X(8, 256, 4, 3, 0, 1) X(8, 256, 4, 1, 0, 1)
#define LUMEN_SHAPES(X) LUMEN_SHAPES_0(X) LUMEN_SHAPES_1(X) LUMEN_SHAPES_2(X) LUMEN_SHAPES_3(X) LUMEN_SHAPES_4(X) \
  LUMEN_SHAPES_5(X) LUMEN_SHAPES_6(X) LUMEN_SHAPES_7(X) LUMEN_SHAPES_8(X) LUMEN_SHAPES_9(X)
#define LUMEN_SHAPE_DECL(G, B, M, T, A, N) int launch_shape<G, B, M, T, A, N>(const Launch&, int, cudaStream_t, int);
// part 10: the wavefront's rounds; part 11: the per-photon, query and locate kernels
#define LUMEN_N_PARTS 12

