// The training context behind the C ABI: upstream's openntc::Context
// (libopenntc/libopenntc.cpp) re-built around libontc's kernels.
//
// What is kept from upstream, because results depend on it:
//   * profile constants, feature/mip/level geometry (libopenntc.cpp:289-338, 1209-1227);
//   * one std::mt19937(123) per context, consumed in upstream's order: latents U(-0.1, 0.1)
//     level by level (g0 then g1), Kaiming-uniform W0, W1, Wout (:483-501), then per step
//     bernoulli(0.05), U(0,1), uniform lod, and the tile origins (:564-583);
//   * the schedule: cosine-annealed learning rates, global-step bias correction for the
//     decoder and per-level step counters for the latents (:711-720), latent lock and
//     quantisation at 95 % of the steps (:475, :601-619);
//   * completion: quantise+pack every level, calibrate, int8 per-row weight quantisation
//     into the decoder blob (:799-876).
// What changes: two launches per step (a fused tile kernel and a fused optimiser pass)
// on one stream, the step's draws uploaded in batches ahead of time, no host sync per step,
// quantisation noise generated at the touched latents only, FP64 loss and PSNR sums.
#include <algorithm>
#include <array>
#include <atomic>
#include <bit>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <sys/stat.h>

#include "../../include/ontc.h"
#include "../../include/ontc_debug.h"
#include "image.h"
#include "json.h"
#include "kernels.h"

using namespace ontc;

namespace {

// Device allocations made through DBuf so far, and the one to fail (ontc_debug_fail_device_alloc;
// 0: none): a host-side stand-in for an out-of-memory cudaMalloc.
std::atomic<int64_t> g_dev_allocs{0};
std::atomic<int64_t> g_fail_alloc{0};

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count)
  {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    const int64_t k = ++g_dev_allocs;
    if (k == g_fail_alloc.load()) {
      n = 0;
      return cudaErrorMemoryAllocation;
    }
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      n = 0;
    }
    return e;
  }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

struct Source {
  std::string path, name;
  bool srgb = false, vflip = false;
  int32_t sem = 0;
  int32_t nch = 0;
  int32_t cmap[4] = {-1, -1, -1, -1};
};

int round_up(int n, int k) { return ((n + k - 1) / k) * k; }

float cosine_annealing(float lr_min, float lr_max, int t_max, int t_cur)
{
  // libopenntc.cpp:419-423
  return lr_min + 0.5f * (lr_max - lr_min) * (1.0f + cosf(t_cur * acosf(-1.0f) / t_max));
}

// libopenntc.cpp:445-469: per-row symmetric int8 (round half away from zero), scale*prescale.
void quantize_weights(const float* Wf, int rows, int cols, float prescale, uint32_t* Wq, float* Ws)
{
  for (int i = 0; i < rows; i++) {
    float max_abs = 0.0f;
    for (int j = 0; j < cols; j++) max_abs = std::max(std::abs(Wf[i * cols + j]), max_abs);
    const float scale = (max_abs == 0.0f) ? 1.0f : max_abs / 127.0f;
    Ws[i] = scale * prescale;
    for (int j = 0; j < cols; j += 4) {
      uint32_t pack = 0;
      for (int c = 0; c < 4; c++) {
        const float val = Wf[i * cols + j + c] / scale;
        const int q = std::clamp((int)std::lroundf(val), -128, 127);
        pack |= ((uint32_t)(q & 0xFF) << (c * 8));
      }
      Wq[i * (cols / 4) + (j / 4)] = pack;
    }
  }
}

// The same int8 rows with each row's scale chosen to minimise the row's squared rounding
// error sum_j (w_j - scale * q_j)^2 over scale = beta * max|w| / 127, beta = 1.00, 0.99, .. 0.60
// (clipping the largest weights when that lowers the error); ties keep the larger scale.
// No upstream counterpart (the calibration search below).
void quantize_weights_mse(const float* Wf, int rows, int cols, float prescale, uint32_t* Wq, float* Ws)
{
  for (int i = 0; i < rows; i++) {
    const float* w = Wf + (size_t)i * cols;
    float max_abs = 0.0f;
    for (int j = 0; j < cols; j++) max_abs = std::max(std::abs(w[j]), max_abs);
    float best = (max_abs == 0.0f) ? 1.0f : max_abs / 127.0f;
    if (max_abs != 0.0f) {
      double best_err = -1.0;
      for (int k = 0; k <= 40; k++) {
        const float scale = (1.0f - 0.01f * (float)k) * max_abs / 127.0f;
        double err = 0.0;
        for (int j = 0; j < cols; j++) {
          const int q = std::clamp((int)std::lroundf(w[j] / scale), -128, 127);
          const double r = (double)w[j] - (double)scale * q;
          err += r * r;
        }
        if (best_err < 0.0 || err < best_err) {
          best_err = err;
          best = scale;
        }
      }
    }
    Ws[i] = best * prescale;
    for (int j = 0; j < cols; j += 4) {
      uint32_t pack = 0;
      for (int c = 0; c < 4; c++) {
        const int q = std::clamp((int)std::lroundf(w[j + c] / best), -128, 127);
        pack |= ((uint32_t)(q & 0xFF) << (c * 8));
      }
      Wq[i * (cols / 4) + (j / 4)] = pack;
    }
  }
}

// libopenntc.cpp:1103-1121
bool valid_semantic_channels(int32_t sem, const std::string& ch)
{
  static const char* rgba = "RGBA";
  if (ch.empty() || ch.size() > 4) return false;
  int p = 0;
  for (char c : ch) {
    while (p < 4 && rgba[p] != c) p++;
    if (p >= 4) return false;
    p++;
  }
  if (sem != 0 && ontc_channel_count_for_semantic(sem) != (int)ch.size()) return false;
  return true;
}

uint32_t step_seed(uint32_t step)
{
  // splitmix-style scramble of the step index: distinct noise streams per step
  uint32_t z = step * 0x9E3779B9u + 0x4F4E5443u;
  z = (z ^ (z >> 16)) * 0x85EBCA6Bu;
  z = (z ^ (z >> 13)) * 0xC2B2AE35u;
  return z ^ (z >> 16);
}

}  // namespace

// The cell rectangles (half-open {x0, y0, x1, y1}) a step's tiles touch in each pyramid, before
// they are merged into a disjoint cover (FootRec); kept per step so consecutive steps'
// footprints can be intersected and subtracted.
struct FootIn {
  int n[2] = {0, 0};
  int r[2][4 * kMaxGrids][4] = {};
  bool whole[2] = {false, false};  // the cover fell back to the whole level
};

struct ontc_context {
  bool initialized = false;
  bool manifest_loaded = false;
  int32_t train_phase = ONTC_MANIFEST_LOADED;
  int last_error = ONTC_SUCCESS;
  int min_dimension = ONTC_MIN_DIMENSION;

  // profile
  int32_t profile = 0, b0 = 0, b1 = 0, C0 = 0, C1 = 0, scale = 0;
  float d0 = 0.f, d1 = 0.f;
  int32_t F = 0, Fp = 0, C = 0, nW = 0;

  // geometry
  int32_t mips = 0, levels = 0;
  int32_t mip_dim[ONTC_MAX_MIPS] = {};
  int32_t g0_dim[ONTC_MAX_LEVELS] = {}, g1_dim[ONTC_MAX_LEVELS] = {};

  // training run
  int32_t batch_count = 0, batch_i = 0, lock_i = 0, grids = 1;
  int32_t grid_batch_i[ONTC_MAX_LEVELS] = {};
  int32_t precision = ONTC_PRECISION_BF16;
  int32_t noise_mode = ONTC_NOISE_COUNTER;
  int32_t optimizer = ONTC_LATENT_ADAM_DEFERRED;
  int32_t calibration = ONTC_CALIBRATION_UPSTREAM;
  bool exact_grad = false;  // ontc_debug_exact_gradients
  int32_t upd_count[ONTC_MAX_LEVELS] = {};  // level steps with a latent update (before the lock)
  int32_t swept[ONTC_MAX_LEVELS] = {};      // every cell of the level has received this many
  int32_t lock_from[ONTC_MAX_LEVELS] = {}, lock_to[ONTC_MAX_LEVELS] = {};  // sweeps at the lock
  uint32_t last_seed = 0;
  bool last_noise = false;
  std::mt19937 gen{123};

  // device
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sms = 148;
  int max_grid = 148;
  DBuf<float> lat[2][4][ONTC_MAX_LEVELS];  // [g0/g1][p,m,v,g][level]
  DBuf<float> W, Wm, Wv, dWpart, calib;
  DBuf<double> loss_part, losses, eval_sums;
  DBuf<StepRec> steps, aux_steps;
  DBuf<int32_t> applied[2][ONTC_MAX_LEVELS];
  DBuf<float4> hist;
  FootRec* h_foots = nullptr;  // pinned staging
  std::vector<FootIn> foot_in;  // per step of the chunk
  // The deferred optimiser's work that the next tile kernel does not read (the next step's
  // catch-up outside this step's footprint, this step's update outside the next one's) runs
  // on `side`, at the lowest priority, beside the tile kernels; events order it.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_pre = nullptr, ev_tile = nullptr, ev_cu = nullptr, ev_side = nullptr;
  bool side_pending = false;
  // tile autotuner (shared batch launches): cost of one unit round of the tcgen05 tile kernel
  // per lod, in microseconds; 0 until tuned
  float unit_us[ONTC_MAX_MIPS] = {};
  DBuf<uint8_t> package[ONTC_MAX_MIPS];
  DBuf<uint32_t> packbuf;
  LatentBoxes boxes[ONTC_MAX_MIPS] = {};  // the tile kernel's TMA staging per lod
  DBuf<int> tc_error;
  DBuf<uint8_t> noise_states;   // upstream-mode cuRAND states (initialised once per context)
  DBuf<float> noise_buf[2];     // upstream-mode level noise buffers, level-0 sized
  static constexpr int kNoiseStates = 1 << 20;  // libopenntc.cpp:377 rand_dim_
  StepRec* h_steps = nullptr;  // pinned staging
  size_t h_steps_cap = 0;

  // host outputs (libopenntc.h:201-210)
  std::vector<uint32_t> g0_host_packed, g1_host_packed;
  uint32_t* g0_host[ONTC_MAX_LEVELS] = {};
  uint32_t* g1_host[ONTC_MAX_LEVELS] = {};
  std::vector<uint8_t> decoder_host;
  ontc_calibration caldata = {};
  Source sources[ONTC_MAX_SOURCES];
  int32_t source_count = 0;
  std::vector<uint8_t> mips_host[ONTC_MAX_SOURCES][ONTC_MAX_MIPS];

  int64_t launches = 0;
  int64_t texels_trained = 0;
  StepRec last_step = {};

  // optional per-kernel timing (ontc_profile_kernels): CUDA events around each launch on
  // the context's stream, reduced when ontc_kernel_times is called
  struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    double bytes, flops;
  };
  bool profiling = false;
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> event_pool;
  cudaEvent_t prof_a = nullptr;
  cudaEvent_t get_event()
  {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void prof_begin(cudaStream_t on = nullptr)
  {
    if (!profiling) return;
    prof_a = get_event();
    cudaEventRecord(prof_a, on ? on : stream);
  }
  void prof_end(int cls, double bytes, double flops, cudaStream_t on = nullptr)
  {
    if (!profiling || !prof_a) return;
    cudaEvent_t b = get_event();
    cudaEventRecord(b, on ? on : stream);
    prof.push_back({cls, prof_a, b, bytes, flops});
    prof_a = nullptr;
  }
  std::vector<float> last_dW;  // decoder gradient of the last ontc_debug_gradients

  Model model() const
  {
    Model M = {};
    M.C0 = C0;
    M.C1 = C1;
    M.F = F;
    M.Fp = Fp;
    M.C = C;
    M.mips = mips;
    M.levels = levels;
    for (int i = 0; i < mips; i++) {
      M.mip_dim[i] = mip_dim[i];
      M.package[i] = package[i].p;
    }
    for (int g = 0; g < 2; g++) {
      Pyramid& P = g == 0 ? M.g0 : M.g1;
      for (int l = 0; l < levels; l++) {
        P.p[l] = lat[g][0][l].p;
        P.m[l] = lat[g][1][l].p;
        P.v[l] = lat[g][2][l].p;
        P.g[l] = lat[g][3][l].p;
        P.dim[l] = g == 0 ? g0_dim[l] : g1_dim[l];
      }
      P.channels = g == 0 ? C0 : C1;
      P.bits = g == 0 ? b0 : b1;
      P.delta = g == 0 ? d0 : d1;
    }
    M.W = W.p;
    M.Wm = Wm.p;
    M.Wv = Wv.p;
    M.nW = nW;
    M.noise0 = noise_buf[0].p;
    M.noise1 = noise_buf[1].p;
    for (int l = 0; l < levels; l++) {
      M.applied[0][l] = applied[0][l].p;
      M.applied[1][l] = applied[1][l].p;
      M.hist[l] = hist.p ? hist.p + (size_t)l * kHistRing : nullptr;
    }
    return M;
  }

  size_t level_elems(int g, int l) const
  {
    const size_t d = (size_t)(g == 0 ? g0_dim[l] : g1_dim[l]);
    return d * d * (size_t)(g == 0 ? C0 : C1);
  }

  int32_t feature_level_for_lod(int32_t lod) const
  {
    // libopenntc.cpp:881-891
    const int first = (int)log2f((float)scale) + 2;
    if (lod < first) return 0;
    return std::min(1 + (lod - first) / 2, levels - 1);
  }
};

namespace {

// Sweep interval in level steps (measured: intervals of 8-64 level steps give the same step time
// at 2048^2).  A cell lags its level by at most this many steps; the hist ring holds twice as
// many so entries written up to a batch of steps ahead never overwrite one a replay reads.
constexpr int kSweepEvery = 64;
static_assert(kHistRing >= 2 * kSweepEvery, "hist entries are written ahead of their updates");

bool ensure_host_steps(ontc_context* c, size_t n)
{
  if (c->h_steps_cap >= n) return true;
  if (c->h_steps) cudaFreeHost(c->h_steps);
  if (c->h_foots) cudaFreeHost(c->h_foots);
  c->h_steps = nullptr;
  c->h_foots = nullptr;
  c->h_steps_cap = 0;
  if (cudaMallocHost(&c->h_steps, n * sizeof(StepRec)) != cudaSuccess) return false;
  if (cudaMallocHost(&c->h_foots, n * sizeof(FootRec)) != cudaSuccess) return false;
  c->h_steps_cap = n;
  return true;
}

// Cell ranges of one pyramid touched by texel range [o, o + T) of a D-wide mip (wrapping),
// with a one-cell margin: the corner cells come from gather_geometry's arithmetic.
void foot_ranges(int o, int T, int D, int gd, int out[2][2], int& n)
{
  auto cells = [&](int a, int b, int* r) {
    const float rm = 1.0f / (float)D;  // exact: D is a power of two
    const int lo = (int)std::floor(((float)a + 0.5f) * rm * (float)gd - 0.5f);
    const int hi = (int)std::floor(((float)b + 0.5f) * rm * (float)gd - 0.5f) + 1;
    r[0] = std::clamp(lo - 1, 0, gd - 1);
    r[1] = std::clamp(hi + 1, 0, gd - 1);
  };
  if (T >= D) {
    cells(0, D - 1, out[0]);
    n = 1;
  } else if (o + T <= D) {
    cells(o, o + T - 1, out[0]);
    n = 1;
  } else {
    cells(o, D - 1, out[0]);
    cells(0, o + T - 1 - D, out[1]);
    n = 2;
  }
}

// Disjoint cover of the cells selected from two sets of half-open rectangles {x0, y0, x1, y1}:
// kCoverUnion the cells in some rectangle of a; kCoverInter those also in some rectangle of b;
// kCoverMinus those in a and in no rectangle of b.  Elementary cells lie between consecutive
// distinct edges of both sets; runs of selected cells are merged along x within each band, and
// runs identical to the previous band's along y.  Returns the count, or -1 past cap.
enum { kCoverUnion = 0, kCoverInter = 1, kCoverMinus = 2 };
int cover_op(const int (*a)[4], int na, const int (*b)[4], int nb, int op, int (*out)[4], int cap)
{
  if (op == kCoverUnion) nb = 0;
  std::vector<int> xs, ys;
  for (int pass = 0; pass < 2; pass++) {
    const int (*r)[4] = pass == 0 ? a : b;
    for (int k = 0; k < (pass == 0 ? na : nb); k++) {
      xs.push_back(r[k][0]);
      xs.push_back(r[k][2]);
      ys.push_back(r[k][1]);
      ys.push_back(r[k][3]);
    }
  }
  std::sort(xs.begin(), xs.end());
  xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
  std::sort(ys.begin(), ys.end());
  ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
  const int nx = (int)xs.size() - 1, ny = (int)ys.size() - 1;
  if (nx <= 0 || ny <= 0) return 0;
  // bit 1: inside a rectangle of a; bit 2: inside one of b
  std::vector<uint8_t> mark((size_t)nx * ny, 0);
  auto paint = [&](const int* r, uint8_t bit) {
    const int ix0 = (int)(std::lower_bound(xs.begin(), xs.end(), r[0]) - xs.begin());
    const int ix1 = (int)(std::lower_bound(xs.begin(), xs.end(), r[2]) - xs.begin());
    const int iy0 = (int)(std::lower_bound(ys.begin(), ys.end(), r[1]) - ys.begin());
    const int iy1 = (int)(std::lower_bound(ys.begin(), ys.end(), r[3]) - ys.begin());
    for (int iy = iy0; iy < iy1; iy++)
      for (int ix = ix0; ix < ix1; ix++) mark[(size_t)iy * nx + ix] |= bit;
  };
  for (int k = 0; k < na; k++) paint(a[k], 1);
  for (int k = 0; k < nb; k++) paint(b[k], 2);
  const uint8_t want = op == kCoverInter ? 3 : 1;
  struct Open { int ix0, ix1, band, out; };
  std::vector<Open> open;
  int m = 0;
  for (int iy = 0; iy < ny; iy++) {
    auto covered = [&](int ix) { return mark[(size_t)iy * nx + ix] == want || (op == kCoverUnion && mark[(size_t)iy * nx + ix]); };
    int ix = 0;
    while (ix < nx) {
      if (!covered(ix)) {
        ix++;
        continue;
      }
      int ix1 = ix + 1;
      while (ix1 < nx && covered(ix1)) ix1++;
      bool extended = false;
      for (Open& o : open)
        if (o.band == iy - 1 && o.ix0 == ix && o.ix1 == ix1) {
          out[o.out][3] = ys[iy + 1];
          o.band = iy;
          extended = true;
          break;
        }
      if (!extended) {
        if (m >= cap) return -1;
        out[m][0] = xs[ix];
        out[m][1] = ys[iy];
        out[m][2] = xs[ix1];
        out[m][3] = ys[iy + 1];
        open.push_back({ix, ix1, iy, m});
        m++;
      }
      ix = ix1;
    }
  }
  return m;
}

// Disjoint cover of the union of in[0..n).
int disjoint_cover(const int (*in)[4], int n, int (*out)[4], int cap)
{
  return cover_op(in, n, nullptr, 0, kCoverUnion, out, cap);
}

// Pyramid g of F from a disjoint rectangle list.
void fill_foot(FootRec& F, int g, const int (*out)[4], int m)
{
  int cells = 0;
  for (int k = 0; k < m; k++) {
    F.r[g][k][0] = (int16_t)out[k][0];
    F.r[g][k][1] = (int16_t)out[k][1];
    F.r[g][k][2] = (int16_t)(out[k][2] - out[k][0]);
    F.r[g][k][3] = (int16_t)(out[k][3] - out[k][1]);
    F.start[g][k] = cells;
    cells += (out[k][2] - out[k][0]) * (out[k][3] - out[k][1]);
  }
  F.n[g] = m;
  F.cells[g] = cells;
}

// The footprint of a step (FootRec, common.cuh): per pyramid the disjoint cover of every
// tile's cell rectangles, or the whole level when the cover needs too many rectangles.
void make_foot(const ontc_context* c, const StepRec& s, FootRec& F, FootIn& fi)
{
  F = FootRec();
  fi = FootIn();
  for (int g = 0; g < 2; g++) {
    const int gd = g == 0 ? c->g0_dim[s.level] : c->g1_dim[s.level];
    int (*in)[4] = fi.r[g];
    int out[kMaxFootRects][4], n = 0;
    for (int t = 0; t < s.n_grids; t++) {
      int xr[2][2], yr[2][2], nx, ny;
      foot_ranges(s.ox[t], s.tile_dim, s.mip_dim, gd, xr, nx);
      foot_ranges(s.oy[t], s.tile_dim, s.mip_dim, gd, yr, ny);
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
          in[n][0] = xr[i][0];
          in[n][1] = yr[j][0];
          in[n][2] = xr[i][1] + 1;
          in[n][3] = yr[j][1] + 1;
          n++;
        }
    }
    fi.n[g] = n;
    int m = disjoint_cover(in, n, out, kMaxFootRects);
    if (m < 0) {
      out[0][0] = out[0][1] = 0;
      out[0][2] = out[0][3] = gd;
      m = 1;
      fi.whole[g] = true;
    }
    fill_foot(F, g, out, m);
  }
}

// For consecutive latent-updating steps a -> b: `cross` = cells of both footprints (updated
// for a before b's tile kernel), `rest` = a's cells outside b (updated for a beside b's tile
// kernel), `ahead` = b's cells outside a (caught up for b beside a's tile kernel).  Steps on
// different levels share no cell.  False when a cover needs more than kMaxFootRects rectangles
// or a footprint fell back to the whole level.
bool split_feet(const StepRec& sa, const FootRec& fa, const FootIn& ia, const StepRec& sb, const FootRec& fb,
                const FootIn& ib, FootRec& cross, FootRec& rest, FootRec& ahead)
{
  cross = FootRec();
  if (sa.level != sb.level) {
    rest = fa;
    ahead = fb;
    return true;
  }
  rest = FootRec();
  ahead = FootRec();
  for (int g = 0; g < 2; g++) {
    if (ia.whole[g] || ib.whole[g]) return false;
    int out[kMaxFootRects][4];
    int m = cover_op(ia.r[g], ia.n[g], ib.r[g], ib.n[g], kCoverInter, out, kMaxFootRects);
    if (m < 0) return false;
    fill_foot(cross, g, out, m);
    m = cover_op(ia.r[g], ia.n[g], ib.r[g], ib.n[g], kCoverMinus, out, kMaxFootRects);
    if (m < 0) return false;
    fill_foot(rest, g, out, m);
    m = cover_op(ib.r[g], ib.n[g], ia.r[g], ia.n[g], kCoverMinus, out, kMaxFootRects);
    if (m < 0) return false;
    fill_foot(ahead, g, out, m);
  }
  return true;
}

// Brings every latent of every level from level step from[l] up to to[l] (deferred optimiser).
cudaError_t sweep_levels(ontc_context* c, const int32_t* from, const int32_t* to)
{
  const Model M = c->model();
  for (int l = 0; l < c->levels; l++) {
    if (to[l] <= from[l]) continue;
    c->prof_begin();
    cudaError_t e = launch_sweep(M, l, from[l], to[l], c->stream);
    c->prof_end(ONTC_KCLASS_CATCHUP, 24.0 * (double)(c->level_elems(0, l) + c->level_elems(1, l)), 0.0);
    c->launches++;
    if (e) return e;
  }
  return cudaSuccess;
}

// Brings every latent of every level up to its level's step count (deferred optimiser).
cudaError_t flush_latents(ontc_context* c)
{
  if (c->optimizer != ONTC_LATENT_ADAM_DEFERRED) return cudaSuccess;
  cudaError_t e = sweep_levels(c, c->swept, c->upd_count);
  for (int l = 0; l < c->levels; l++) c->swept[l] = c->upd_count[l];
  return e;
}

// Full-mip "step" used by Eval and Calibrate: every texel of the mip once.
StepRec full_mip_rec(const ontc_context* c, int mip)
{
  StepRec s = {};
  s.lod = mip;
  s.level = c->feature_level_for_lod(mip);
  s.mip_dim = c->mip_dim[mip];
  s.tile_dim = c->mip_dim[mip];
  s.n_grids = 1;
  s.texels = c->mip_dim[mip] * c->mip_dim[mip];
  // upstream's Eval/Calibrate add whatever its noise buffers hold (zero after the lock)
  s.noise = c->noise_mode == ONTC_NOISE_UPSTREAM ? 2 : (c->last_noise ? 1 : 0);
  s.seed = c->last_seed;
  s.norm_lod = mip / static_cast<float>(c->mips - 1);
  s.step = 0;
  return s;
}

// Releases everything a manifest holds, also the buffers of a load that failed part way.
void unload(ontc_context* c)
{
  for (int g = 0; g < 2; g++)
    for (int k = 0; k < 4; k++)
      for (int l = 0; l < ONTC_MAX_LEVELS; l++) c->lat[g][k][l].release();
  for (int i = 0; i < ONTC_MAX_MIPS; i++) c->package[i].release();
  c->packbuf.release();
  c->losses.release();
  c->noise_buf[0].release();
  c->noise_buf[1].release();
  for (int g = 0; g < 2; g++)
    for (int l = 0; l < ONTC_MAX_LEVELS; l++) c->applied[g][l].release();
  c->hist.release();
  c->g0_host_packed.clear();
  c->g1_host_packed.clear();
  for (int i = 0; i < ONTC_MAX_LEVELS; i++) c->g0_host[i] = c->g1_host[i] = nullptr;
  for (int s = 0; s < ONTC_MAX_SOURCES; s++)
    for (int m = 0; m < ONTC_MAX_MIPS; m++) c->mips_host[s][m].clear();
  c->manifest_loaded = false;
}

// The tensor-core kernel reports a bounded-wait timeout through this word instead of
// spinning; the context treats it as a CUDA failure.
bool tc_failed(ontc_context* c)
{
  int flag = 0;
  if (cudaMemcpy(&flag, c->tc_error.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return true;
  return flag != 0;
}

ontc_train_progress make_progress(int32_t phase, int32_t result, const ontc_context* c)
{
  ontc_train_progress p = {};
  p.phase = phase;
  p.result = result;
  p.batches_complete = c->batch_i;
  p.total_batches = c->batch_count;
  return p;
}

// Runs the forward over every texel of every mip (Eval / Calibrate, libopenntc.cpp:898-1053).
cudaError_t full_forward(ontc_context* c, int mode, std::vector<double>* sums)
{
  const Model M = c->model();
  for (int mip = 0; mip < c->mips; mip++) c->h_steps[mip] = full_mip_rec(c, mip);
  cudaError_t e = cudaMemcpyAsync(c->aux_steps.p, c->h_steps, c->mips * sizeof(StepRec), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return e;
  if (mode == kCalib) {
    e = cudaMemsetAsync(c->calib.p, 0, 2 * sizeof(float), c->stream);
    if (e != cudaSuccess) return e;
  }
  for (int mip = 0; mip < c->mips; mip++) {
    const int units = (c->mip_dim[mip] * c->mip_dim[mip] + kTile - 1) / kTile;
    const int grid = std::min(units, c->sms);
    TileOut out = {c->dWpart.p, c->loss_part.p, c->calib.p};
    e = launch_simt_units(mode, M, c->aux_steps.p, mip, grid, out, c->stream);
    c->launches++;
    if (e != cudaSuccess) return e;
    if (mode == kEval) {
      e = launch_sum_doubles(c->loss_part.p, grid, c->eval_sums.p + mip, c->stream);
      c->launches++;
      if (e != cudaSuccess) return e;
    }
  }
  if (mode == kEval) {
    sums->assign(c->mips, 0.0);
    e = cudaMemcpyAsync(sums->data(), c->eval_sums.p, c->mips * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaStreamSynchronize(c->stream);
}

ontc_calibration calibrate(ontc_context* c, float headroom, cudaError_t* err)
{
  ontc_calibration cal = {};
  *err = full_forward(c, kCalib, nullptr);
  if (*err != cudaSuccess) return cal;
  float hmax[2] = {0.f, 0.f};
  *err = cudaMemcpy(hmax, c->calib.p, sizeof(hmax), cudaMemcpyDeviceToHost);
  if (*err != cudaSuccess) return cal;
  cal.max_abs_a1 = hmax[0];
  cal.max_abs_a2 = hmax[1];
  cal.s_a1 = headroom * hmax[0] / 127.0f;
  cal.s_a2 = headroom * hmax[1] / 127.0f;
  return cal;
}

// The int8 decoder blob (libopenntc.cpp:841-876; layout DEC_*_OFFSET, ntc_decode.hlsli:95-103)
// from the fp32 weights Wh with activation scales s_a1, s_a2: upstream's per-row max scales
// (QuantizeWeights) or, with mse_weights, the per-row squared-error-optimal ones.
void build_blob(const ontc_context* c, const std::vector<float>& Wh, float s_a1, float s_a2, bool mse_weights,
                uint8_t* out)
{
  const int H = kHidden;
  std::vector<float> W0pad((size_t)H * c->Fp, 0.0f);
  for (int i = 0; i < H; i++) memcpy(&W0pad[(size_t)i * c->Fp], &Wh[(size_t)i * c->F], c->F * sizeof(float));
  uint8_t* dec = out;
  uint32_t* W0q = (uint32_t*)dec;
  dec += H * c->Fp;
  uint32_t* W1q = (uint32_t*)dec;
  dec += H * H;
  uint32_t* Woq = (uint32_t*)dec;
  dec += kOutPad * H;
  float* W0s = (float*)dec;
  dec += H * sizeof(float);
  float* W1s = (float*)dec;
  dec += H * sizeof(float);
  float* Wos = (float*)dec;
  const auto q = mse_weights ? quantize_weights_mse : quantize_weights;
  q(W0pad.data(), H, c->Fp, 1.0f / 128.0f, W0q, W0s);
  q(&Wh[w1_off(c->F)], H, H, s_a1, W1q, W1s);
  q(&Wh[wo_off(c->F)], c->C, H, s_a2, Woq, Wos);
  memset(Woq + c->C * (H / 4), 0, (size_t)(kOutPad - c->C) * H);
  for (int i = c->C; i < kOutPad; i++) Wos[i] = 0.0f;
}

// The context's mip chain and training targets as decode-evaluation texels.
TexelMap texel_map(const ontc_context* c)
{
  TexelMap m;
  m.mips = c->mips;
  m.C = c->C;
  for (int i = 0; i < c->mips; i++) {
    m.dim[i] = c->mip_dim[i];
    m.target[i] = c->package[i].p;
    m.start[i + 1] = m.start[i] + (int64_t)c->mip_dim[i] * c->mip_dim[i];
  }
  return m;
}

// Device scratch of a decoded evaluation: `chunk` samples (uv, lod, outputs), fixed-grid
// block partials and one fp64 sum per chunk.
struct EvalScratch {
  static constexpr int kBlocks = 512;
  DBuf<float> uv, out;
  DBuf<int32_t> lod;
  DBuf<double> partial, sums;
  cudaError_t alloc(int64_t chunk, int C, int chunks)
  {
    cudaError_t e = uv.alloc((size_t)chunk * 2);
    if (!e) e = lod.alloc((size_t)chunk);
    if (!e) e = out.alloc((size_t)chunk * C);
    if (!e) e = partial.alloc(kBlocks);
    if (!e) e = sums.alloc((size_t)chunks);
    return e;
  }
};

// sums[slot] = squared decode error of samples [j0, j0 + n) whose uv/lod are in the scratch.
cudaError_t decode_sq_err(ontc_context* c, ontc_decoder* dec, const TexelMap& m, int64_t j0, int64_t n,
                          EvalScratch& s, int slot)
{
  if (ontc_decode(dec, s.uv.p, s.lod.p, n, s.out.p) != ONTC_SUCCESS) return cudaErrorLaunchFailure;
  cudaError_t e = launch_decoded_sq_err(m, j0, n, s.out.p, s.partial.p, EvalScratch::kBlocks, c->stream);
  if (!e) e = launch_sum_doubles(s.partial.p, EvalScratch::kBlocks, s.sums.p + slot, c->stream);
  c->launches += 3;
  return e;
}

// A decoder of the context's completed material (latents as packed, current blob).
cudaError_t context_decoder(ontc_context* c, ontc_decoder** dec)
{
  ontc_compressed_data cd;
  ontc_get_compressed_data(c, &cd);
  const int r = ontc_decoder_create(&cd, ONTC_DECODE_INT8, c->stream, dec);
  return r == ONTC_SUCCESS ? cudaSuccess : (r == ONTC_ALLOCATION_FAILURE ? cudaErrorMemoryAllocation : cudaErrorUnknown);
}

// Squared decode error summed over every texel of every mip, in chunks of 4 M samples.
cudaError_t decoded_sq_err_all(ontc_context* c, double* sum)
{
  ontc_decoder* dec = nullptr;
  cudaError_t e = context_decoder(c, &dec);
  if (e != cudaSuccess) return e;
  const TexelMap m = texel_map(c);
  const int64_t total = m.start[m.mips];
  const int64_t chunk = std::min<int64_t>(total, 1 << 22);
  const int chunks = (int)((total + chunk - 1) / chunk);
  EvalScratch s;
  e = s.alloc(chunk, c->C, chunks);
  for (int k = 0; k < chunks && e == cudaSuccess; k++) {
    const int64_t j0 = (int64_t)k * chunk, n = std::min(chunk, total - j0);
    e = launch_texel_samples(m, j0, n, s.uv.p, s.lod.p, c->stream);
    c->launches++;
    if (!e) e = decode_sq_err(c, dec, m, j0, n, s, k);
  }
  std::vector<double> sums(chunks, 0.0);
  if (!e) e = cudaMemcpyAsync(sums.data(), s.sums.p, chunks * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (!e && ontc_decoder_status(dec) != ONTC_SUCCESS) e = cudaErrorLaunchFailure;
  ontc_decoder_destroy(dec);
  *sum = 0.0;
  for (double v : sums) *sum += v;
  return e;
}

struct Calib {
  float s_a1 = 0.0f, s_a2 = 0.0f;
  bool mse_weights = false;
};

// ONTC_CALIBRATION_SEARCH (no upstream counterpart): the activation scales and the weight
// rounding scales that minimise the int8 decode's squared error against the targets on a
// fixed sample of up to 2^21 texels spread over every mip.  Coordinate descent over
// s_a1 = a1 * s_a1(upstream), s_a2 = a2 * s_a2(upstream), a in {1, 0.8, 0.8^2, .., 0.8^10},
// twice, then per-row weight scales (max or squared-error-optimal); upstream's choice
// (a1 = a2 = 1, max weights) is the first candidate, so the result never scores worse on the
// sample.  The blob layout and file format are unchanged.
cudaError_t search_calibration(ontc_context* c, const std::vector<float>& Wh, Calib* best_out)
{
  const float base1 = c->caldata.s_a1, base2 = c->caldata.s_a2;
  ontc_decoder* dec = nullptr;
  cudaError_t e = context_decoder(c, &dec);
  if (e != cudaSuccess) return e;
  TexelMap m = texel_map(c);
  const int64_t total = m.start[m.mips];
  const int64_t n = std::min<int64_t>(total, 1 << 21);
  if (n < total) {
    int64_t stride = 2654435761ll;  // odd, > total: coprime once the gcd is 1
    while (std::gcd(stride, total) != 1) stride += 2;
    m.stride = stride;
  }
  EvalScratch s;
  e = s.alloc(n, c->C, 1);
  if (!e) e = launch_texel_samples(m, 0, n, s.uv.p, s.lod.p, c->stream);
  c->launches++;
  std::vector<uint8_t> blob(c->decoder_host.size());
  auto score = [&](float a1, float a2, bool mw, double* err) -> cudaError_t {
    build_blob(c, Wh, a1 * base1, a2 * base2, mw, blob.data());
    if (ontc::decoder_set_weights(dec, blob.data(), blob.size(), a1 * base1, a2 * base2) != ONTC_SUCCESS)
      return cudaErrorUnknown;
    cudaError_t r = decode_sq_err(c, dec, m, 0, n, s, 0);
    if (!r) r = cudaMemcpyAsync(err, s.sums.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (!r) r = cudaStreamSynchronize(c->stream);
    return r;
  };
  float a[11];
  a[0] = 1.0f;
  for (int i = 1; i < 11; i++) a[i] = a[i - 1] * 0.8f;
  float b1 = 1.0f, b2 = 1.0f;
  bool bw = false;
  double best = 0.0;
  if (!e) e = score(b1, b2, bw, &best);
  for (int pass = 0; pass < 2 && !e; pass++)
    for (int axis = 0; axis < 2 && !e; axis++)
      for (int i = 0; i < 11 && !e; i++) {
        const float t1 = axis == 0 ? a[i] : b1, t2 = axis == 1 ? a[i] : b2;
        if (t1 == b1 && t2 == b2) continue;
        double err = 0.0;
        e = score(t1, t2, bw, &err);
        if (!e && err < best) {
          best = err;
          b1 = t1;
          b2 = t2;
        }
      }
  if (!e) {
    double err = 0.0;
    e = score(b1, b2, true, &err);
    if (!e && err < best) bw = true;
  }
  if (!e && ontc_decoder_status(dec) != ONTC_SUCCESS) e = cudaErrorLaunchFailure;
  ontc_decoder_destroy(dec);
  best_out->s_a1 = b1 * base1;
  best_out->s_a2 = b2 * base2;
  best_out->mse_weights = bw;
  return e;
}

// Training completion (libopenntc.cpp:799-876).
cudaError_t complete_training(ontc_context* c)
{
  cudaError_t e;
  for (int l = 0; l < c->levels; l++) {
    for (int g = 0; g < 2; g++) {
      const size_t n = c->level_elems(g, l);
      const int bits = g == 0 ? c->b0 : c->b1;
      e = launch_quantize_pack(c->lat[g][0][l].p, (long long)n, bits, c->packbuf.p, c->stream);
      c->launches++;
      if (e != cudaSuccess) return e;
      uint32_t* dst = g == 0 ? c->g0_host[l] : c->g1_host[l];
      e = cudaMemcpyAsync(dst, c->packbuf.p, n * bits / 8, cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) return e;
      e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess) return e;
    }
  }
  c->caldata = calibrate(c, 1.1f, &e);
  if (e != cudaSuccess) return e;

  std::vector<float> Wh(c->nW);
  e = cudaMemcpy(Wh.data(), c->W.p, c->nW * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  build_blob(c, Wh, c->caldata.s_a1, c->caldata.s_a2, false, c->decoder_host.data());
  if (c->calibration == ONTC_CALIBRATION_SEARCH && c->caldata.s_a1 > 0.0f && c->caldata.s_a2 > 0.0f) {
    Calib best;
    e = search_calibration(c, Wh, &best);
    if (e != cudaSuccess) return e;
    c->caldata.s_a1 = best.s_a1;
    c->caldata.s_a2 = best.s_a2;
    build_blob(c, Wh, best.s_a1, best.s_a2, best.mse_weights, c->decoder_host.data());
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

ontc_context* ontc_create(void) { return new ontc_context(); }

void ontc_destroy(ontc_context* c)
{
  if (!c) return;
  unload(c);
  if (c->h_steps) cudaFreeHost(c->h_steps);
  if (c->h_foots) cudaFreeHost(c->h_foots);
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
  }
  for (cudaEvent_t ev : {c->ev_pre, c->ev_tile, c->ev_cu, c->ev_side})
    if (ev) cudaEventDestroy(ev);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int ontc_init(ontc_context* c, int32_t profile, void* stream)
{
  if (c->initialized) return ONTC_INVALID_STATE;
  c->profile = profile;
  switch (profile) {  // libopenntc.cpp:289-318
    case ONTC_BPP_0_2: c->b0 = 2; c->b1 = 4; c->C0 = 8; c->C1 = 12; break;
    case ONTC_BPP_0_5: c->b0 = 4; c->b1 = 4; c->C0 = 12; c->C1 = 20; break;
    case ONTC_BPP_1_0: c->b0 = 2; c->b1 = 4; c->C0 = 12; c->C1 = 10; break;
    case ONTC_BPP_2_25: c->b0 = 4; c->b1 = 4; c->C0 = 16; c->C1 = 12; break;
    default: return ONTC_INVALID_STATE;
  }
  c->scale = (profile == ONTC_BPP_1_0 || profile == ONTC_BPP_2_25) ? 2 : 4;
  c->d0 = 2.0f / powf(2.0f, (float)c->b0);
  c->d1 = 2.0f / powf(2.0f, (float)c->b1);
  c->F = round_up(4 * c->C0 + c->C1 + 12 + 1, 4);
  c->Fp = round_up(c->F, 16);
  c->nW = n_weights(c->F);

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ONTC_CUDA_FAILURE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ONTC_CUDA_FAILURE;
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
  c->max_grid = std::max(c->sms, std::max(1, tc_max_grid()));
  if (stream) {
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
  } else {
    // the library's own stream at the highest priority: the tile kernels and the work they wait
    // for go before the side stream's (lowest priority) whenever both have CTAs pending
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, greatest) != cudaSuccess)
      return ONTC_CUDA_FAILURE;
    c->own_stream = true;
  }
  if (c->W.alloc(c->nW) || c->Wm.alloc(c->nW) || c->Wv.alloc(c->nW) || c->dWpart.alloc((size_t)c->max_grid * c->nW) ||
      c->loss_part.alloc(c->max_grid) || c->calib.alloc(2) || c->eval_sums.alloc(ONTC_MAX_MIPS) ||
      c->aux_steps.alloc(ONTC_MAX_MIPS) || c->tc_error.alloc(4) || !ensure_host_steps(c, 1024)) {
    // a failed Init holds nothing: it can be retried, or the context destroyed
    for (auto* b : {&c->W, &c->Wm, &c->Wv, &c->dWpart}) b->release();
    c->loss_part.release();
    c->calib.release();
    c->aux_steps.release();
    c->tc_error.release();
    c->eval_sums.release();
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = nullptr;
    c->own_stream = false;
    return ONTC_ALLOCATION_FAILURE;
  }
  cudaMemset(c->W.p, 0, c->nW * sizeof(float));
  cudaMemset(c->dWpart.p, 0, c->nW * sizeof(float));  // the accumulated gradient row starts at zero
  cudaMemset(c->tc_error.p, 0, 4 * sizeof(int));
  const size_t dec = (size_t)kHidden * c->Fp + kHidden * kHidden + kOutPad * kHidden + kHidden * 4 + kHidden * 4 +
                     kOutPad * 4;  // libopenntc.cpp:381-387
  c->decoder_host.assign(dec, 0);
  c->initialized = true;
  return ONTC_SUCCESS;
}

int ontc_set_min_dimension(ontc_context* c, int32_t dim)
{
  if (dim < 16 || dim > ONTC_MAX_DIMENSION || std::popcount((unsigned)dim) != 1) return ONTC_INVALID_DIMENSION;
  c->min_dimension = dim;
  return ONTC_SUCCESS;
}

void ontc_unload_manifest(ontc_context* c) { unload(c); }

int ontc_load_manifest(ontc_context* c, const char* path)
{
  unload(c);
  std::ifstream f(path, std::ios::binary);
  if (!f) return ONTC_FILE_NOT_FOUND;
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  Json j;
  if (!Json::parse(text.data(), text.data() + text.size(), j) || !j.is_object() || !j.find("textures"))
    return ONTC_INVALID_MANIFEST;
  auto int_or = [](const Json& o, const char* k, int64_t d, bool& ok) -> int64_t {
    const Json* v = o.find(k);
    if (!v) return d;
    if (!v->is_number()) {
      ok = false;
      return d;
    }
    return v->as_int();
  };
  bool ok = true;
  const int64_t width = int_or(j, "width", -1, ok), height = int_or(j, "height", -1, ok);
  if (!ok) return ONTC_INVALID_MANIFEST;
  if (width == -1 && height == -1) return ONTC_INVALID_MANIFEST;
  if (width != -1 && height != -1 && width != height) return ONTC_INVALID_MANIFEST;
  const int64_t dim = width == -1 ? height : width;
  if (dim < c->min_dimension || dim > ONTC_MAX_DIMENSION) return ONTC_INVALID_MANIFEST;

  const Json& texs = *j.find("textures");
  std::vector<const Json*> tlist;
  if (texs.is_array()) {
    for (const Json& t : texs.items()) tlist.push_back(&t);
  } else if (texs.is_object()) {
    for (const auto& kv : texs.members()) tlist.push_back(&kv.second);
  } else {
    tlist.push_back(&texs);
  }
  int count = 0;
  for (const Json* t : tlist) {
    const Json* sems = t->find("semantics");
    const Json* fname = t->find("fileName");
    if (!sems || !sems->is_object()) return ONTC_INVALID_MANIFEST;
    if (!fname || !fname->is_string()) return ONTC_INVALID_MANIFEST;
    for (const auto& kv : sems->members()) {  // key order, as nlohmann's std::map iterates
      if (!kv.second.is_string()) return ONTC_INVALID_MANIFEST;
      const int32_t sem = ontc_semantic_from_name(kv.first.c_str());
      const std::string& chs = kv.second.as_string();
      if (!valid_semantic_channels(sem, chs)) return ONTC_INVALID_MANIFEST;
      if (count >= ONTC_MAX_SOURCES) return ONTC_INVALID_MANIFEST;
      Source& s = c->sources[count];
      s = Source();
      s.path = fname->as_string();
      const Json* nm = t->find("name");
      if (nm && nm->is_string()) s.name = nm->as_string();
      const Json* sr = t->find("isSRGB");
      const Json* vf = t->find("verticalFlip");
      if ((sr && !sr->is_bool()) || (vf && !vf->is_bool())) return ONTC_INVALID_MANIFEST;
      s.srgb = sr ? sr->as_bool() : false;  // parsed but unused, as upstream (:1164)
      s.vflip = vf ? vf->as_bool() : false;
      s.sem = sem;
      s.nch = ontc_channel_count_for_semantic(sem);
      // an unknown semantic name has no channel count (upstream carries -1 on into its totals,
      // allocations and launches when valid sources make the total positive): rejected here
      if (s.nch < 1) return ONTC_INVALID_MANIFEST;
      for (int i = 0; i < 4; i++) {
        int ch = -1;
        if (i < s.nch) ch = chs[i] == 'R' ? 0 : chs[i] == 'G' ? 1 : chs[i] == 'B' ? 2 : 3;
        s.cmap[i] = ch;
      }
      count++;
    }
  }
  c->source_count = count;
  int total = 0;
  for (int i = 0; i < count; i++) total += c->sources[i].nch;
  if (total < 1 || total > ONTC_MAX_CHANNELS) return ONTC_INVALID_MANIFEST;
  c->C = total;
  std::stable_sort(c->sources, c->sources + count, [](const Source& a, const Source& b) { return a.sem < b.sem; });
  if (dim < c->min_dimension || dim > ONTC_MAX_DIMENSION || std::popcount((unsigned)dim) != 1) return ONTC_INVALID_DIMENSION;
  // manifest validation above needs no device; everything below does
  if (!c->initialized) return ONTC_INVALID_STATE;

  // mip and latent pyramids (libopenntc.cpp:1209-1227)
  c->mip_dim[0] = (int)dim;
  c->mips = 0;
  while (c->mip_dim[c->mips] > 4) {
    c->mip_dim[c->mips + 1] = c->mip_dim[c->mips] / 2;
    c->mips++;
  }
  c->mips++;
  c->levels = 0;
  c->g0_dim[0] = c->mip_dim[0] / c->scale;
  c->g1_dim[0] = c->g0_dim[0] / 2;
  while (c->g0_dim[c->levels] / 4 >= 4) {
    c->g0_dim[c->levels + 1] = c->g0_dim[c->levels] / 4;
    c->g1_dim[c->levels + 1] = c->g1_dim[c->levels] / 4;
    c->levels++;
  }
  c->levels++;

  c->manifest_loaded = true;  // so that unload() releases partial allocations
  auto fail = [&](int r) {
    unload(c);
    return r;
  };
  size_t words0 = 0, words1 = 0;
  for (int l = 0; l < c->levels; l++) {
    for (int g = 0; g < 2; g++) {
      const size_t n = c->level_elems(g, l);
      for (int k = 0; k < 4; k++)
        if (c->lat[g][k][l].alloc(n) != cudaSuccess) return fail(ONTC_ALLOCATION_FAILURE);
      cudaMemsetAsync(c->lat[g][3][l].p, 0, n * sizeof(float), c->stream);
    }
    words0 += c->level_elems(0, l) * c->b0 / 32;
    words1 += c->level_elems(1, l) * c->b1 / 32;
    if (c->applied[0][l].alloc((size_t)c->g0_dim[l] * c->g0_dim[l]) ||
        c->applied[1][l].alloc((size_t)c->g1_dim[l] * c->g1_dim[l]))
      return fail(ONTC_ALLOCATION_FAILURE);
  }
  if (c->hist.alloc((size_t)c->levels * kHistRing)) return fail(ONTC_ALLOCATION_FAILURE);
  if (c->packbuf.alloc(std::max(c->level_elems(0, 0) * c->b0 / 32, c->level_elems(1, 0) * c->b1 / 32) + 4))
    return fail(ONTC_ALLOCATION_FAILURE);
  // TMA staging boxes of each lod's level (no staging where the driver cannot encode tensor maps)
  for (int m = 0; m < c->mips; m++) {
    const int l = c->feature_level_for_lod(m);
    const cudaError_t be = make_latent_boxes(c->lat[0][0][l].p, c->lat[1][0][l].p, c->g0_dim[l], c->g1_dim[l], c->C0,
                                             c->C1, c->mip_dim[m], tc_box_capacity(), c->boxes[m]);
    if (be == cudaErrorNotSupported) {
      for (int j = 0; j < c->mips; j++) c->boxes[j].w0 = 0;
      break;
    }
    if (be != cudaSuccess) return fail(ONTC_CUDA_FAILURE);
  }
  c->g0_host_packed.assign(words0, 0);
  c->g1_host_packed.assign(words1, 0);
  size_t o0 = 0, o1 = 0;
  for (int l = 0; l < c->levels; l++) {
    c->g0_host[l] = c->g0_host_packed.data() + o0;
    c->g1_host[l] = c->g1_host_packed.data() + o1;
    o0 += c->level_elems(0, l) * c->b0 / 32;
    o1 += c->level_elems(1, l) * c->b1 / 32;
  }
  for (int m = 0; m < c->mips; m++)
    if (c->package[m].alloc((size_t)c->mip_dim[m] * c->mip_dim[m] * c->C)) return fail(ONTC_ALLOCATION_FAILURE);

  // Mip chains per source (libopenntc.cpp:1296-1336)
  const size_t n0 = (size_t)dim * dim;
  DBuf<uint8_t> rgba_dev;
  std::vector<DBuf<uint8_t>> src_mips((size_t)count * c->mips);
  if (rgba_dev.alloc(n0 * 4)) return fail(ONTC_ALLOCATION_FAILURE);
  int pkg_off = 0;  // the source's first channel in the target package (sources in package order)
  std::string base_dir;
  {
    std::string p(path);
    const size_t sl = p.find_last_of('/');
    if (sl != std::string::npos) base_dir = p.substr(0, sl + 1);
  }
  for (int i = 0; i < count; i++) {
    const Source& s = c->sources[i];
    std::vector<uint8_t> rgba;
    int w = 0, h = 0;
    bool loaded = load_image_rgba8(s.path, rgba, w, h);
    // extension: relative paths that do not resolve from the working directory are
    // also tried relative to the manifest's directory
    if (!loaded && !s.path.empty() && s.path[0] != '/' && !base_dir.empty())
      loaded = load_image_rgba8(base_dir + s.path, rgba, w, h);
    if (!loaded) return fail(ONTC_FILE_NOT_FOUND);
    if (w != h || w != dim) return fail(ONTC_INVALID_MANIFEST);
    if (s.nch < 1) continue;  // a semantic with no channel count contributes no channels
    if (cudaMemcpyAsync(rgba_dev.p, rgba.data(), n0 * 4, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
      return fail(ONTC_CUDA_FAILURE);
    for (int m = 0; m < c->mips; m++)
      if (src_mips[(size_t)i * c->mips + m].alloc((size_t)c->mip_dim[m] * c->mip_dim[m] * s.nch))
        return fail(ONTC_ALLOCATION_FAILURE);
    // the chain fused with packaging: each mip of this source is written once, into the
    // source's mip and into its channels of that mip's target package (libopenntc.cpp:1338-1362)
    if (launch_prepare_package(rgba_dev.p, (int)dim, s.cmap, s.nch, src_mips[(size_t)i * c->mips].p, c->package[0].p,
                               c->C, pkg_off, c->stream))
      return fail(ONTC_CUDA_FAILURE);
    c->launches++;
    for (int m = 1; m < c->mips; m++) {
      if (launch_lanczos_down_package(src_mips[(size_t)i * c->mips + m - 1].p, c->mip_dim[m - 1], s.nch,
                                      src_mips[(size_t)i * c->mips + m].p, c->package[m].p, c->C, pkg_off, c->stream))
        return fail(ONTC_CUDA_FAILURE);
      c->launches++;
    }
    pkg_off += s.nch;
    for (int m = 0; m < c->mips; m++) {
      c->mips_host[i][m].assign((size_t)c->mip_dim[m] * c->mip_dim[m] * s.nch, 0);
      if (cudaMemcpyAsync(c->mips_host[i][m].data(), src_mips[(size_t)i * c->mips + m].p, c->mips_host[i][m].size(),
                          cudaMemcpyDeviceToHost, c->stream))
        return fail(ONTC_CUDA_FAILURE);
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(ONTC_CUDA_FAILURE);
  }
  if (pkg_off != c->C) return fail(ONTC_INVALID_MANIFEST);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(ONTC_CUDA_FAILURE);
  c->train_phase = ONTC_MANIFEST_LOADED;
  return ONTC_SUCCESS;
}

void ontc_begin_training(ontc_context* c, int32_t quality, int32_t grids_per_batch)
{
  if (!c->manifest_loaded ||
      (c->train_phase != ONTC_MANIFEST_LOADED && c->train_phase != ONTC_TRAIN_COMPLETE &&
       c->train_phase != ONTC_TRAIN_IN_PROGRESS && c->train_phase != ONTC_TRAIN_ERROR)) {
    c->last_error = ONTC_INVALID_STATE;
    return;
  }
  c->batch_count = ontc_steps_for_quality(quality);
  c->lock_i = (95 * c->batch_count) / 100;
  c->batch_i = 0;
  c->grids = std::clamp(grids_per_batch, 1, kMaxGrids);
  for (int l = 0; l < ONTC_MAX_LEVELS; l++) c->grid_batch_i[l] = c->upd_count[l] = c->swept[l] = 0;
  if (!deferred_supported(c->C0, c->C1)) c->optimizer = ONTC_LATENT_ADAM_DENSE;
  c->last_noise = false;

  cudaError_t e = cudaSuccess;
  std::vector<float> tmp;
  std::uniform_real_distribution<float> lat(-0.1f, 0.1f);
  for (int l = 0; l < c->levels; l++) {
    for (int g = 0; g < 2; g++) {
      const size_t n = c->level_elems(g, l);
      tmp.resize(n);
      for (size_t i = 0; i < n; i++) tmp[i] = lat(c->gen);
      if (!e) e = cudaMemcpy(c->lat[g][0][l].p, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice);
      if (!e) e = cudaMemset(c->lat[g][1][l].p, 0, n * sizeof(float));
      if (!e) e = cudaMemset(c->lat[g][2][l].p, 0, n * sizeof(float));
      if (!e) e = cudaMemset(c->lat[g][3][l].p, 0, n * sizeof(float));
      if (!e) e = cudaMemset(c->applied[g][l].p, 0, c->applied[g][l].n * sizeof(int32_t));
    }
  }
  // Kaiming-uniform, bound 1/sqrt(fan_in) (libopenntc.cpp:60-78): W0 [64][F], W1 [64][64], Wout [16][64]
  tmp.assign(c->nW, 0.0f);
  auto kaiming = [&](float* dst, int rows, int cols) {
    const float bound = 1.0f / sqrtf((float)cols);
    std::uniform_real_distribution<float> d(-bound, bound);
    for (int i = 0; i < rows * cols; i++) dst[i] = d(c->gen);
  };
  kaiming(&tmp[0], kHidden, c->F);
  kaiming(&tmp[w1_off(c->F)], kHidden, kHidden);
  kaiming(&tmp[wo_off(c->F)], kOutPad, kHidden);
  if (!e) e = cudaMemcpy(c->W.p, tmp.data(), c->nW * sizeof(float), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemset(c->Wm.p, 0, c->nW * sizeof(float));
  if (!e) e = cudaMemset(c->Wv.p, 0, c->nW * sizeof(float));
  if (!e) e = cudaMemset(c->dWpart.p, 0, c->nW * sizeof(float));  // after a tile kernel that stopped early
  if (!e) e = c->losses.alloc((size_t)std::max(c->batch_count, 1));
  if (!e) e = cudaMemset(c->losses.p, 0, c->losses.n * sizeof(double));
  // a failed start (no step-loss buffer, a failed upload) leaves the context in TrainError: no
  // step may run on it until ontc_begin_training succeeds
  if (e) c->last_error = e == cudaErrorMemoryAllocation ? ONTC_ALLOCATION_FAILURE : ONTC_CUDA_FAILURE;
  c->train_phase = e ? ONTC_TRAIN_ERROR : ONTC_TRAIN_IN_PROGRESS;
}

int ontc_set_train_options(ontc_context* c, const ontc_train_options* o)
{
  if (!c->initialized || !o) return ONTC_INVALID_STATE;
  if (o->precision != ONTC_PRECISION_FP32 && o->precision != ONTC_PRECISION_BF16 && o->precision != ONTC_PRECISION_BF16X3)
    return ONTC_INVALID_STATE;
  if (c->batch_i > 0) return ONTC_INVALID_STATE;
  if (o->noise_mode != ONTC_NOISE_COUNTER && o->noise_mode != ONTC_NOISE_UPSTREAM) return ONTC_INVALID_STATE;
  if (o->latent_adam != ONTC_LATENT_ADAM_DEFERRED && o->latent_adam != ONTC_LATENT_ADAM_DENSE) return ONTC_INVALID_STATE;
  if (o->calibration != ONTC_CALIBRATION_UPSTREAM && o->calibration != ONTC_CALIBRATION_SEARCH) return ONTC_INVALID_STATE;
  if (o->noise_mode == ONTC_NOISE_UPSTREAM && !c->manifest_loaded) return ONTC_INVALID_STATE;
  // a buffer the options need that cannot be had leaves the context in TrainError (no step may
  // run with a missing step-loss or noise buffer) until ontc_begin_training succeeds again
  auto fail = [&](int r) {
    c->last_error = r;
    if (c->manifest_loaded) c->train_phase = ONTC_TRAIN_ERROR;
    return r;
  };
  c->precision = o->precision;
  if (o->steps_override > 0) {
    c->batch_count = o->steps_override;
    c->lock_i = (95 * c->batch_count) / 100;
    if (c->manifest_loaded) {
      if (c->losses.alloc((size_t)c->batch_count)) return fail(ONTC_ALLOCATION_FAILURE);
      if (cudaMemset(c->losses.p, 0, c->losses.n * sizeof(double))) return fail(ONTC_CUDA_FAILURE);
    }
  }
  if (o->has_lock_step) c->lock_i = std::max(0, o->lock_step);
  c->calibration = o->calibration;
  // the deferred kernels are compiled per profile channel pair; anything else runs dense
  c->optimizer = deferred_supported(c->C0, c->C1) ? o->latent_adam : ONTC_LATENT_ADAM_DENSE;
  if (o->noise_mode == ONTC_NOISE_UPSTREAM) {
    if (!c->noise_states.p) {
      if (c->noise_states.alloc(noise_state_bytes(ontc_context::kNoiseStates))) return fail(ONTC_ALLOCATION_FAILURE);
      if (launch_noise_init(c->noise_states.p, ontc_context::kNoiseStates, c->stream)) return fail(ONTC_CUDA_FAILURE);
      c->launches++;
    }
    for (int g = 0; g < 2; g++) {
      if (!c->noise_buf[g].p) {
        if (c->noise_buf[g].alloc(c->level_elems(g, 0))) return fail(ONTC_ALLOCATION_FAILURE);
        if (cudaMemsetAsync(c->noise_buf[g].p, 0, c->noise_buf[g].n * sizeof(float), c->stream))
          return fail(ONTC_CUDA_FAILURE);
      }
    }
  }
  c->noise_mode = o->noise_mode;  // set once its buffers exist
  return ONTC_SUCCESS;
}

// Context::Train (libopenntc.cpp:536-879)
}  // extern "C"

namespace {

// Draws and enqueues the next chunk of steps toward `target` (at most 1024, ending before the
// lock step so that the latents can be snapped first); returns without waiting for the GPU.
// Makes `side` (lowest priority) and its events on first use.
cudaError_t ensure_side(ontc_context* c)
{
  if (c->side) return cudaSuccess;
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (!e) e = cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, least);
  for (cudaEvent_t* ev : {&c->ev_pre, &c->ev_tile, &c->ev_cu, &c->ev_side})
    if (!e) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  return e;
}

// Orders everything enqueued on `side` so far before what is enqueued on the main stream next.
cudaError_t drain_side(ontc_context* c)
{
  if (!c->side_pending) return cudaSuccess;
  c->side_pending = false;
  cudaError_t e = cudaEventRecord(c->ev_side, c->side);
  if (!e) e = cudaStreamWaitEvent(c->stream, c->ev_side, 0);
  return e;
}

// Steps a chunk draws and enqueues at most (one slot each in the step records).
constexpr int kChunkCap = 1024;

// Per latent-updating step k of the deferred optimiser, when step k + 1 updates latents too
// and needs no level sweep first (footprints F(k), F(k+1)):
//   main: [catch-up of F(k) outside F(k-1): done on side] -> tile(k) -> decoder Adam + update
//         of F(k) -> tile(k+1) ...
//   side: catch-up of F(k+1) \ F(k), after the step records are uploaded (it runs as SMs free
//         up: beside the end of tile(k) and the update of F(k)).
// The side kernel touches no latent the concurrent tile kernel or main-stream update reads or
// writes, and every cell's updates and replays keep their order (a cell of F(k+1) \ F(k) was
// last updated before tile(k)), so the values are those of the serial schedule bit for bit.
// Otherwise step k runs serially on the main stream after the side stream drains.
// One chunk of steps of one context, enqueued step by step: begin(), then per batch of up to
// kPrepBatch steps prep(), and per step pre() (everything before the step's tile launch),
// tile() (the context's own launch) and post() (everything after), then end().  enqueue_chunk
// runs it alone; ontc_train_batch runs several in lock step around shared tile launches.
struct ChunkRun {
  static constexpr int kPrepBatch = 8;
  ontc_context* c = nullptr;
  std::bernoulli_distribution dist_batch_type{0.05};
  std::uniform_real_distribution<float> dist_u{0.0f, 1.0f};
  std::uniform_int_distribution<int> dist_lod;
  Model M{};
  int first = 0, cnt = 0;
  int drawn = 0, uploaded = 0;
  int ahead_step = -1;  // the step whose catch-up was enqueued on side
  bool deferred_mode = false;
  cudaError_t e = cudaSuccess;
  // the step between pre() and post()
  FootRec cross{}, rest{}, next_cu{};
  bool look = false, deferred = false;
  int grid = 0, cls = ONTC_KCLASS_UNITS_FP32;
  int pre_k = -1;  // the last step pre() began
  // the side stream's lookahead (next catch-up beside the tile, the update outside the next
  // footprint after it); without it each step's catch-up and update run on the main stream
  bool lookahead = true;

  // Waits for the context's previous chunk and sizes this one: at most `cap` steps toward
  // `target`, ending at the lock step.
  cudaError_t begin(ontc_context* ctx, int target, int cap)
  {
    c = ctx;
    dist_lod = std::uniform_int_distribution<int>(0, c->mips - 1);
    M = c->model();
    // The previous chunk's kernels may still read the staging and device records.
    e = cudaStreamSynchronize(c->stream);
    if (e) return e;
    first = c->batch_i;
    cnt = std::min(cap, target - first);
    // a chunk ends at the lock step so the latents can be snapped before it runs
    if (first < c->lock_i && first + cnt > c->lock_i) cnt = c->lock_i - first;
    if ((int)c->foot_in.size() < kChunkCap) c->foot_in.resize(kChunkCap);
    deferred_mode = c->optimizer == ONTC_LATENT_ADAM_DEFERRED;
    if (deferred_mode && !e) e = ensure_side(c);
    return e;
  }

  // Steps are drawn in order, one ahead of the batch being launched (a step's lookahead needs
  // the next footprint), uploaded and launched kPrepBatch at a time, so the GPU starts after
  // the first few and the host prepares the rest while it runs (every step has its own slot).
  void prep(int k0, int k1)
  {
    (void)k0;
    if (e) return;
    for (int k = drawn; k < std::min(cnt, k1 + 1); k++) {
      const int bi = first + k;
      const bool draw_uniform = dist_batch_type(c->gen);
      const float U = dist_u(c->gen);
      const float fl = std::floor(0.5f * -std::log2(U));
      int lod = (fl < 1e9f) ? std::min((int)fl, c->mips - 1) : c->mips - 1;
      const int lod_uniform = dist_lod(c->gen);
      if (draw_uniform) lod = lod_uniform;
      StepRec& s = c->h_steps[k];
      s = StepRec();
      s.lod = lod;
      s.level = c->feature_level_for_lod(lod);
      s.mip_dim = c->mip_dim[lod];
      std::uniform_int_distribution<int> dist_grid(0, c->mip_dim[lod] - 1);
      for (int g = 0; g < c->grids; g++) {
        s.ox[g] = dist_grid(c->gen);
        s.oy[g] = dist_grid(c->gen);
      }
      s.tile_dim = std::min(c->mip_dim[lod], 256);
      s.n_grids = c->grids;
      s.texels = c->grids * s.tile_dim * s.tile_dim;
      s.noise = bi < c->lock_i ? (c->noise_mode == ONTC_NOISE_UPSTREAM ? 2 : 1) : 0;
      s.grid_update = bi < c->lock_i ? 1 : 0;
      s.seed = step_seed((uint32_t)bi);
      s.norm_lod = lod / static_cast<float>(c->mips - 1);
      s.b1 = 1.0f / (1.0f - powf(0.9f, bi + 1.0f));
      s.b2 = 1.0f / (1.0f - powf(0.999f, bi + 1.0f));
      s.gb1 = 1.0f / (1.0f - powf(0.9f, c->grid_batch_i[s.level] + 1.0f));
      s.gb2 = 1.0f / (1.0f - powf(0.999f, c->grid_batch_i[s.level] + 1.0f));
      c->grid_batch_i[s.level] += 1;
      // deferred optimiser bookkeeping, in step order: the floor each level is swept to
      s.gstep = c->upd_count[s.level];
      s.gfloor = 0;
      s.sweep_from = -1;
      if (bi == c->lock_i && c->optimizer == ONTC_LATENT_ADAM_DEFERRED)
        for (int l = 0; l < c->levels; l++) {
          c->lock_from[l] = c->swept[l];
          c->lock_to[l] = c->upd_count[l];
          c->swept[l] = c->upd_count[l];
        }
      if (s.grid_update) {
        c->upd_count[s.level] += 1;
        if (c->optimizer == ONTC_LATENT_ADAM_DEFERRED) {
          // a cell may lag its level by at most kSweepEvery steps: the level is swept every
          // kSweepEvery level steps
          if (s.gstep - c->swept[s.level] >= kSweepEvery) {
            s.sweep_from = c->swept[s.level];
            c->swept[s.level] = s.gstep;
          }
          s.gfloor = c->swept[s.level];
          make_foot(c, s, c->h_foots[k], c->foot_in[k]);
        }
      }
      s.exact_grad = c->exact_grad ? 1 : 0;
      s.lr_grid = cosine_annealing(0.0f, 0.01f, c->batch_count, bi);
      // the exact-gradient test mode holds the decoder fixed: the two tile groups of a CTA add
      // their weight-gradient products to shared TMEM accumulators in arrival order, so the
      // decoder gradient is not bit-reproducible from run to run
      s.lr_dec = c->exact_grad ? 0.0f : cosine_annealing(0.0f, 0.005f, c->batch_count, bi);
      s.step = bi;
    }
    drawn = std::max(drawn, std::min(cnt, k1 + 1));
    e = cudaMemcpyAsync(c->steps.p + uploaded, c->h_steps + uploaded, (drawn - uploaded) * sizeof(StepRec),
                        cudaMemcpyHostToDevice, c->stream);
    if (!e && deferred_mode) {
      e = launch_hist_write(M, c->steps.p, uploaded, drawn, c->stream);
      c->launches++;
    }
    uploaded = drawn;
  }

  void pre(int k)
  {
    if (e) return;
    pre_k = k;
    const int bi = first + k;
    const StepRec& s = c->h_steps[k];
    const bool ahead = ahead_step == k;
    if (!ahead) e = drain_side(c);
    if (!e && c->noise_mode == ONTC_NOISE_UPSTREAM && bi < c->lock_i) {
      // upstream regenerates the step level's noise buffers before every step (libopenntc.cpp:586-600)
      for (int g = 0; g < 2 && e == cudaSuccess; g++)
        e = launch_noise_fill(c->noise_states.p, ontc_context::kNoiseStates, (long long)c->level_elems(g, s.level),
                              g == 0 ? c->d0 : c->d1, c->noise_buf[g].p, c->stream);
      c->launches += 2;
    }
    if (!e && bi == c->lock_i) {
      // one-time snap of every level to its integer lattice (libopenntc.cpp:601-619)
      if (deferred_mode) e = sweep_levels(c, c->lock_from, c->lock_to);
      for (int l = 0; l < c->levels && e == cudaSuccess; l++) {
        e = launch_quantize_grid(c->lat[0][0][l].p, (long long)c->level_elems(0, l), c->b0, c->d0, c->stream);
        if (!e) e = launch_quantize_grid(c->lat[1][0][l].p, (long long)c->level_elems(1, l), c->b1, c->d1, c->stream);
        c->launches += 2;
      }
      for (int g = 0; g < 2 && e == cudaSuccess; g++)
        if (c->noise_buf[g].p) e = cudaMemsetAsync(c->noise_buf[g].p, 0, c->noise_buf[g].n * sizeof(float), c->stream);
    }
    deferred = deferred_mode && s.grid_update;
    const FootRec& fr = c->h_foots[k];
    if (deferred && !ahead) {
      if (s.sweep_from >= 0) {
        c->prof_begin();
        if (!e) e = launch_sweep(M, s.level, s.sweep_from, s.gstep, c->stream);
        c->prof_end(ONTC_KCLASS_CATCHUP, 24.0 * (double)(c->level_elems(0, s.level) + c->level_elems(1, s.level)),
                    0.0);
        c->launches++;
      }
      c->prof_begin();
      if (!e) e = launch_catchup(M, c->steps.p, k, fr, false, c->stream);
      // reads and writes p, m, v of the footprint latents that lag
      c->prof_end(ONTC_KCLASS_CATCHUP, 24.0 * ((double)fr.cells[0] * c->C0 + (double)fr.cells[1] * c->C1), 0.0);
      c->launches++;
    }
    if (ahead && !e) e = cudaStreamWaitEvent(c->stream, c->ev_cu, 0);
    // the next step's catch-up outside this footprint, on side beside this tile kernel
    look = false;
    if (lookahead && deferred && k + 1 < drawn) {
      const StepRec& n = c->h_steps[k + 1];
      look = n.grid_update && n.sweep_from < 0 &&
             split_feet(s, fr, c->foot_in[k], n, c->h_foots[k + 1], c->foot_in[k + 1], cross, rest, next_cu);
    }
    if (look && !e) {
      e = cudaEventRecord(c->ev_pre, c->stream);  // after the record uploads and this step's catch-up
      if (!e) e = cudaStreamWaitEvent(c->side, c->ev_pre, 0);
      c->prof_begin(c->side);
      if (!e) e = launch_catchup(M, c->steps.p, k + 1, next_cu, true, c->side);
      c->prof_end(ONTC_KCLASS_SIDE_CATCHUP,
                  24.0 * ((double)next_cu.cells[0] * c->C0 + (double)next_cu.cells[1] * c->C1), 0.0, c->side);
      c->launches++;
      if (!e) e = cudaEventRecord(c->ev_cu, c->side);
      ahead_step = k + 1;
      c->side_pending = true;
    }
  }

  void tile(int k)
  {
    const StepRec& s = c->h_steps[k];
    const int units = (s.texels + kTile - 1) / kTile;
    TileOut to = {c->dWpart.p, c->loss_part.p, nullptr};
    grid = std::min(units, c->sms);
    cls = ONTC_KCLASS_UNITS_FP32;
    c->prof_begin();
    if (e) {
    } else if (c->precision == ONTC_PRECISION_BF16 || c->precision == ONTC_PRECISION_BF16X3) {
      const bool split = c->precision == ONTC_PRECISION_BF16X3;
      const int gpc = tc_groups_per_cta(split);  // work units in flight per CTA
      grid = std::min((units + gpc - 1) / gpc, tc_max_grid());
      cls = split ? ONTC_KCLASS_UNITS_BF16X3 : ONTC_KCLASS_UNITS_BF16;
      e = launch_tc_units(M, c->steps.p, k, grid, to, c->tc_error.p, c->boxes[s.lod], split, c->stream);
      if (e == cudaErrorNotSupported) {
        cudaGetLastError();
        grid = std::min(units, c->sms);
        cls = ONTC_KCLASS_UNITS_FP32;
        e = launch_simt_units(kTrain, M, c->steps.p, k, grid, to, c->stream);
      }
    } else {
      e = launch_simt_units(kTrain, M, c->steps.p, k, grid, to, c->stream);
    }
    // MLP fwd + both backward GEMMs per texel: 3 x 2 x (64 F + 64*64 + 64 C) flops
    c->prof_end(cls, (double)s.texels * c->C, 6.0 * (double)s.texels * (64.0 * c->F + 4096.0 + 64.0 * c->C));
    c->launches++;
  }

  void post(int k)
  {
    const int bi = first + k;
    const StepRec& s = c->h_steps[k];
    const FootRec& fr = c->h_foots[k];
    // the tcgen05 tile kernels add every CTA's decoder gradient into row 0 of dWpart
    const bool dw_acc = cls != ONTC_KCLASS_UNITS_FP32;
    if (deferred) {
      // the whole footprint on the main stream, beside the next step's catch-up on side (they
      // touch disjoint cells); a tile CTA fills its SM's register file, so an update left for
      // the side stream would only run between tile launches anyway
      c->prof_begin();
      if (!e)
        e = launch_footprint_update(M, c->steps.p, k, fr, true, c->dWpart.p, dw_acc, c->loss_part.p, grid, c->losses.p,
                                    c->stream);
      // footprint latents: p, m, v, g in and out (32 B each)
      c->prof_end(ONTC_KCLASS_ADAM, 32.0 * ((double)fr.cells[0] * c->C0 + (double)fr.cells[1] * c->C1), 0.0);
      c->launches++;
    } else {
      c->prof_begin();
      if (!e) e = launch_adam_step(M, c->steps.p, k, c->dWpart.p, dw_acc, c->loss_part.p, grid, c->losses.p, c->stream);
      // latent Adam streams p, m, v, g in and out once: 32 bytes per latent of the level
      c->prof_end(ONTC_KCLASS_ADAM,
                  s.grid_update ? 32.0 * (double)(c->level_elems(0, s.level) + c->level_elems(1, s.level)) : 0.0,
                  0.0);
      c->launches++;
    }
    c->last_seed = s.seed;
    c->last_noise = s.noise != 0;
    c->last_step = s;
    c->texels_trained += s.texels;
    c->batch_i = bi + 1;
  }

  cudaError_t end()
  {
    const cudaError_t d = drain_side(c);
    return e ? e : d;
  }
};

// Draws and enqueues the next chunk of steps (at most kChunkCap, ending at the lock step).
cudaError_t enqueue_chunk(ontc_context* c, int target)
{
  ChunkRun r;
  if (r.begin(c, target, kChunkCap)) return r.e;
  for (int k0 = 0; k0 < r.cnt && r.e == cudaSuccess; k0 += ChunkRun::kPrepBatch) {
    const int k1 = std::min(r.cnt, k0 + ChunkRun::kPrepBatch);
    r.prep(k0, k1);
    for (int k = k0; k < k1 && r.e == cudaSuccess; k++) {
      r.pre(k);
      r.tile(k);
      r.post(k);
    }
  }
  return r.end();
}

// Ends a run of ontc_train chunks: every latent current, the stream drained and checked, the
// progress reported and, at the last step, the completion artefacts built.
void finish_train(ontc_context* c, cudaError_t e, ontc_train_progress* out)
{
  // every latent is current whenever control returns to the caller
  if (!e) e = flush_latents(c);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (!e && tc_failed(c)) e = cudaErrorLaunchTimeout;
  if (e != cudaSuccess) {
    c->last_error = ONTC_CUDA_FAILURE;
    *out = make_progress(ONTC_TRAIN_ERROR, ONTC_CUDA_FAILURE, c);
    return;
  }
  *out = make_progress(ONTC_TRAIN_IN_PROGRESS, ONTC_SUCCESS, c);
  if (c->batch_i == c->batch_count) {
    out->phase = ONTC_TRAIN_COMPLETE;
    c->train_phase = ONTC_TRAIN_COMPLETE;
    if (complete_training(c) != cudaSuccess) {
      c->last_error = ONTC_CUDA_FAILURE;
      *out = make_progress(ONTC_TRAIN_ERROR, ONTC_CUDA_FAILURE, c);
    }
  }
}

}  // namespace

extern "C" {

void ontc_train(ontc_context* c, int32_t num_batches, ontc_train_progress* out)
{
  if (!c->manifest_loaded || (c->train_phase != ONTC_TRAIN_IN_PROGRESS && c->train_phase != ONTC_TRAIN_COMPLETE)) {
    *out = make_progress(ONTC_TRAIN_ERROR, ONTC_INVALID_STATE, c);
    return;
  }
  if (num_batches < 0) num_batches = 0;
  const int remaining = std::max(0, c->batch_count - c->batch_i);
  const int n = std::min(remaining, num_batches);
  const int target = c->batch_i + n;
  if (c->batch_i == target) {
    *out = make_progress(ONTC_TRAIN_COMPLETE, ONTC_SUCCESS, c);
    return;
  }
  if (!ensure_host_steps(c, 1024) || (c->steps.n < (size_t)1024 && c->steps.alloc(1024))) {
    c->last_error = ONTC_CUDA_FAILURE;
    *out = make_progress(ONTC_TRAIN_ERROR, ONTC_CUDA_FAILURE, c);
    return;
  }
  cudaError_t e = cudaSuccess;
  while (c->batch_i < target && e == cudaSuccess) e = enqueue_chunk(c, target);
  finish_train(c, e, out);
}

void ontc_train_until_complete(ontc_context* c, ontc_train_progress* out) { ontc_train(c, c->batch_count, out); }

}  // extern "C"

namespace {

// Steps the next chunk of context c toward `target` holds (as ChunkRun::begin sizes it).
int chunk_steps(const ontc_context* c, int target)
{
  int cnt = std::min(kChunkCap, target - c->batch_i);
  if (c->batch_i < c->lock_i && c->batch_i + cnt > c->lock_i) cnt = c->lock_i - c->batch_i;
  return cnt;
}

// CTAs of a shared tile launch per material: one each, then every further SM to the material
// that takes longest (its unit rounds, units / (gpc x CTAs) rounded up, times its measured
// cost of a round), as long as one still gains from it; the launch lasts as long as its
// longest material.
void partition_ctas(const std::vector<int>& units, const std::vector<float>& cost, int gpc, int sms,
                    std::vector<int>& ctas)
{
  const int n = (int)units.size();
  ctas.assign(n, 1);
  auto time = [&](int i) { return (float)((units[i] + gpc * ctas[i] - 1) / (gpc * ctas[i])) * cost[i]; };
  for (int used = n; used < sms; used++) {
    int best = -1;
    for (int i = 0; i < n; i++) {
      if (ctas[i] * gpc >= units[i]) continue;  // one unit per group already
      if (best < 0 || time(i) > time(best) || (time(i) == time(best) && units[i] > units[best])) best = i;
    }
    if (best < 0) break;
    ctas[best]++;
  }
}

// ---- tile autotuner -------------------------------------------------------------------------
// The cost of one unit round (each group of every CTA through one 128-texel unit) of a
// context's tcgen05 tile kernel, per lod: it depends on the profile shape and on how the lod's
// texels fall on the latent grids (staged boxes or not, separable scatter or not).  Measured by
// timed trial launches of a representative step on scratch gradient buffers (the training
// state is not touched), kept in the context and in a cache file: ONTC_TUNE_CACHE, else
// $XDG_CACHE_HOME or ~/.cache + /openntc_b200/tile_costs.txt (ONTC_TUNE_CACHE="" keeps them in
// memory only).  Lines: "<device>|<C0>,<C1>,<Fp>|<mip>,<d0>,<d1>,<texels> <microseconds>".
std::string tune_cache_path()
{
  if (const char* p = getenv("ONTC_TUNE_CACHE")) return p;
  std::string base;
  if (const char* x = getenv("XDG_CACHE_HOME"); x && *x) base = x;
  else if (const char* h = getenv("HOME"); h && *h) base = std::string(h) + "/.cache";
  else return "";
  return base + "/openntc_b200/tile_costs.txt";
}

std::string tune_key(const ontc_context* c, int lod, const char* device)
{
  const int level = c->feature_level_for_lod(lod), mip = c->mip_dim[lod];
  const int tile = std::min(mip, 256);
  char k[256];
  snprintf(k, sizeof(k), "%s|%d,%d,%d|%d,%d,%d,%d", device, c->C0, c->C1, c->model().Fp, mip, c->g0_dim[level],
           c->g1_dim[level], c->grids * tile * tile);
  for (char* q = k; *q; q++)
    if (*q == ' ') *q = '_';
  return k;
}

cudaError_t tune_tiles(ontc_context* c)
{
  bool done = true;
  for (int l = 0; l < c->mips; l++) done = done && c->unit_us[l] > 0.0f;
  if (done) return cudaSuccess;
  int dev = 0;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDevice(&dev);
  if (!e) e = cudaGetDeviceProperties(&prop, dev);
  if (e) return e;
  // cached costs
  const std::string path = tune_cache_path();
  std::vector<std::pair<std::string, float>> cached;
  if (!path.empty()) {
    std::ifstream f(path);
    std::string key;
    float us;
    while (f >> key >> us) cached.emplace_back(key, us);
  }
  std::vector<int> todo;
  for (int l = 0; l < c->mips; l++) {
    if (c->unit_us[l] > 0.0f) continue;
    const std::string key = tune_key(c, l, prop.name);
    for (const auto& kv : cached)
      if (kv.first == key) c->unit_us[l] = kv.second;
    if (c->unit_us[l] <= 0.0f) todo.push_back(l);
  }
  if (todo.empty()) return cudaSuccess;
  // trials on scratch gradients, losses and error flag
  size_t g0n = 0, g1n = 0;
  for (int l = 0; l < c->levels; l++) {
    g0n = std::max(g0n, c->level_elems(0, l));
    g1n = std::max(g1n, c->level_elems(1, l));
  }
  DBuf<float> g0s, g1s, dws;
  DBuf<double> lps;
  DBuf<int> errs;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  e = cudaStreamSynchronize(c->stream);
  if (!e) e = g0s.alloc(g0n);
  if (!e) e = g1s.alloc(g1n);
  if (!e) e = dws.alloc(c->nW);
  if (!e) e = lps.alloc(c->max_grid);
  if (!e) e = errs.alloc(4);
  if (!e) e = cudaMemsetAsync(errs.p, 0, 4 * sizeof(int), c->stream);
  if (!e) e = cudaEventCreate(&t0);
  if (!e) e = cudaEventCreate(&t1);
  std::vector<StepRec> recs(c->mips);
  for (int l = 0; l < c->mips && !e; l++) {
    StepRec& s = recs[l];
    s = StepRec();
    s.lod = l;
    s.level = c->feature_level_for_lod(l);
    s.mip_dim = c->mip_dim[l];
    s.tile_dim = std::min(s.mip_dim, 256);
    s.n_grids = c->grids;
    s.texels = c->grids * s.tile_dim * s.tile_dim;
    s.noise = 1;
    s.grid_update = 1;
    s.seed = 12345u + (uint32_t)l;
    s.norm_lod = l / static_cast<float>(c->mips - 1);
    for (int g = 0; g < c->grids; g++) {  // spread over the mip, as the uniform draws are
      s.ox[g] = (int)(((int64_t)(2 * g + 1) * s.mip_dim * 37) / 101) % s.mip_dim;
      s.oy[g] = (int)(((int64_t)(2 * g + 1) * s.mip_dim * 59) / 103) % s.mip_dim;
    }
  }
  if (!e) e = cudaMemcpyAsync(c->aux_steps.p, recs.data(), c->mips * sizeof(StepRec), cudaMemcpyHostToDevice, c->stream);
  std::vector<std::string> lines;
  for (int l : todo) {
    if (e) break;
    const StepRec& s = recs[l];
    Model M = c->model();
    M.g0.g[s.level] = g0s.p;
    M.g1.g[s.level] = g1s.p;
    const TileOut to = {dws.p, lps.p, nullptr};
    const int units = (s.texels + kTile - 1) / kTile, gpc = tc_groups_per_cta(false);
    const int grid = std::min((units + gpc - 1) / gpc, tc_max_grid());
    float best = 0.0f;
    for (int rep = 0; rep < 4 && !e; rep++) {  // one warm-up, then the fastest of three
      e = cudaEventRecord(t0, c->stream);
      if (!e) e = launch_tc_units(M, c->aux_steps.p, l, grid, to, errs.p, c->boxes[l], false, c->stream);
      if (!e) e = cudaEventRecord(t1, c->stream);
      if (!e) e = cudaEventSynchronize(t1);
      float ms = 0.0f;
      if (!e) e = cudaEventElapsedTime(&ms, t0, t1);
      c->launches++;
      if (rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    if (e) break;
    const int rounds = (units + gpc * grid - 1) / (gpc * grid);
    c->unit_us[l] = std::max(1e-3f, 1e3f * best / (float)rounds);
    char v[32];
    snprintf(v, sizeof(v), " %.4f", c->unit_us[l]);
    lines.push_back(tune_key(c, l, prop.name) + v);
  }
  if (!e) e = cudaStreamSynchronize(c->stream);
  int flag[4] = {};
  if (!e) e = cudaMemcpy(flag, errs.p, sizeof(flag), cudaMemcpyDeviceToHost);
  if (!e && flag[0]) e = cudaErrorLaunchTimeout;  // a bounded wait gave up: no costs from it
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (e) {
    for (int l : todo) c->unit_us[l] = 0.0f;
    return e;
  }
  if (!path.empty() && !lines.empty()) {
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos) {
      std::string dir = path.substr(0, slash);
      for (size_t i = 1; i <= dir.size(); i++)  // mkdir -p
        if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    std::ofstream f(path, std::ios::app);
    for (const auto& line : lines) f << line << "\n";
  }
  return cudaSuccess;
}

// The streams and events of shared tile launches: a stream per profile shape, an event per
// context (its step's work before the tile) and per shape (the shared tile done).
struct SharedTiles {
  std::vector<cudaStream_t> stream;
  std::vector<cudaEvent_t> ev_tile, ev_pre;
  ~SharedTiles()
  {
    for (cudaStream_t st : stream)
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    for (cudaEvent_t ev : ev_tile) if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : ev_pre) if (ev) cudaEventDestroy(ev);
  }
  cudaError_t init(int n_ctx, int n_shapes)
  {
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    stream.assign(n_shapes, nullptr);
    ev_tile.assign(n_shapes, nullptr);
    ev_pre.assign(n_ctx, nullptr);
    for (auto& st : stream) if (!e) e = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest);
    for (auto& ev : ev_tile) if (!e) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    for (auto& ev : ev_pre) if (!e) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    return e;
  }
};

// Step k of every context in `live` (runs[i] between pre(k) and post(k)) in one tcgen05 tile
// launch per profile shape, each on its own stream: a launch's SMs are split among its
// materials by their measured unit-round costs, and the launches of different shapes share the
// GPU as separate kernels do.  Sets each run's grid and kernel class for its post(k).
void shared_tile_step(ontc_context* const* ctxs, std::vector<ChunkRun>& runs, const std::vector<int>& live,
                      const std::vector<int>& shape_of, SharedTiles& st, int k)
{
  for (int sh = 0; sh < (int)st.stream.size(); sh++) {
    std::vector<int> idx, units, ctas;
    std::vector<float> cost;
    for (int i : live) {
      if (shape_of[i] != sh || runs[i].e != cudaSuccess) continue;
      const StepRec& s = ctxs[i]->h_steps[k];
      idx.push_back(i);
      units.push_back((s.texels + kTile - 1) / kTile);
      const float us = ctxs[i]->unit_us[s.lod];
      cost.push_back(us > 0.0f ? us : 1.0f);
    }
    const int nm = (int)idx.size();
    if (nm == 0) continue;
    partition_ctas(units, cost, tc_groups_per_cta(false), tc_max_grid(), ctas);
    TileMat mats[kMaxTileMats];
    int begin = 0;
    for (int m = 0; m < nm; m++) {
      ontc_context* c = ctxs[idx[m]];
      const StepRec& s = c->h_steps[k];
      TileMat& t = mats[m];
      memset(&t, 0, sizeof(t));
      t.boxes = c->boxes[s.lod];
      t.M = runs[idx[m]].M;
      t.step = c->steps.p + k;
      t.out = TileOut{c->dWpart.p, c->loss_part.p, nullptr};
      t.err = c->tc_error.p;
      t.cta_begin = begin;
      t.cta_count = ctas[m];
      begin += ctas[m];
    }
    cudaError_t e = cudaSuccess;
    for (int m = 0; m < nm && !e; m++) {
      e = cudaEventRecord(st.ev_pre[idx[m]], ctxs[idx[m]]->stream);
      if (!e) e = cudaStreamWaitEvent(st.stream[sh], st.ev_pre[idx[m]], 0);
    }
    // the shared launch counts (and, when profiled, is timed) as a launch of its first material
    ontc_context* c0 = ctxs[idx[0]];
    double bytes = 0.0, flops = 0.0;
    for (int m = 0; m < nm; m++) {
      const ontc_context* c = ctxs[idx[m]];
      const double tex = c->h_steps[k].texels;
      bytes += tex * c->C;
      flops += 6.0 * tex * (64.0 * c->F + 4096.0 + 64.0 * c->C);
    }
    c0->prof_begin(st.stream[sh]);
    if (!e) e = launch_tc_multi(mats, nm, st.stream[sh]);
    c0->prof_end(ONTC_KCLASS_UNITS_BF16, bytes, flops, st.stream[sh]);
    if (!e) e = cudaEventRecord(st.ev_tile[sh], st.stream[sh]);
    c0->launches++;
    for (int m = 0; m < nm; m++) {
      ChunkRun& r = runs[idx[m]];
      if (!e) e = cudaStreamWaitEvent(ctxs[idx[m]]->stream, st.ev_tile[sh], 0);
      r.grid = mats[m].cta_count;
      r.cls = ONTC_KCLASS_UNITS_BF16;
    }
    if (e)
      for (int m = 0; m < nm; m++) runs[idx[m]].e = e;
  }
}

// The contexts of ontc_train_batch advanced in lock step, chunk by chunk, with shared tile
// launches.  err[i] receives each context's outcome.
void train_shared(ontc_context* const* ctxs, const std::vector<int>& target, const std::vector<char>& active,
                  const std::vector<int>& shape_of, int n_shapes, std::vector<cudaError_t>& err)
{
  const int n = (int)target.size();
  SharedTiles st;
  const cudaError_t se = st.init(n, n_shapes);

  // unit-round costs per lod for the SM split (timed once, cached); without them every unit
  // round counts the same
  for (int i = 0; i < n; i++)
    if (active[i] && err[i] == cudaSuccess && !se && tune_tiles(ctxs[i]) != cudaSuccess) cudaGetLastError();
  std::vector<ChunkRun> runs(n);
  for (;;) {
    std::vector<int> live;
    for (int i = 0; i < n; i++)
      if (active[i] && err[i] == cudaSuccess && ctxs[i]->batch_i < target[i]) {
        if (se) err[i] = se;
        else live.push_back(i);
      }
    if (live.empty()) return;
    int cap = kChunkCap;
    for (int i : live) cap = std::min(cap, chunk_steps(ctxs[i], target[i]));
    for (int i : live) {
      runs[i] = ChunkRun();
      // the materials' streams already overlap one another's catch-ups and updates: no side
      // stream (measured on the 16-material set: 1.69 ms per step without, 1.72 with)
      runs[i].lookahead = false;
      runs[i].begin(ctxs[i], target[i], cap);
    }
    for (int k0 = 0; k0 < cap; k0 += ChunkRun::kPrepBatch) {
      const int k1 = std::min(cap, k0 + ChunkRun::kPrepBatch);
      for (int i : live) runs[i].prep(k0, k1);
      for (int k = k0; k < k1; k++) {
        for (int i : live) runs[i].pre(k);
        shared_tile_step(ctxs, runs, live, shape_of, st, k);
        for (int i : live)
          if (runs[i].pre_k == k) runs[i].post(k);
      }
    }
    for (int i : live) err[i] = runs[i].end();
  }
}

}  // namespace

extern "C" {

int ontc_train_batch(ontc_context* const* ctxs, int32_t n, int32_t num_batches, ontc_train_progress* out)
{
  if (n < 0 || (n > 0 && (!ctxs || !out))) return ONTC_INVALID_STATE;
  std::vector<int> target(n, 0);
  std::vector<cudaError_t> err(n, cudaSuccess);
  std::vector<char> active(n, 0);
  for (int i = 0; i < n; i++) {
    ontc_context* c = ctxs[i];
    if (!c) return ONTC_INVALID_STATE;
    for (int j = 0; j < i; j++)
      if (ctxs[j] == c) return ONTC_INVALID_STATE;  // each context once
    if (!c->manifest_loaded || (c->train_phase != ONTC_TRAIN_IN_PROGRESS && c->train_phase != ONTC_TRAIN_COMPLETE)) {
      out[i] = make_progress(ONTC_TRAIN_ERROR, ONTC_INVALID_STATE, c);
      continue;
    }
    const int remaining = std::max(0, c->batch_count - c->batch_i);
    target[i] = c->batch_i + std::min(remaining, std::max(0, num_batches));
    if (target[i] == c->batch_i) {
      out[i] = make_progress(ONTC_TRAIN_COMPLETE, ONTC_SUCCESS, c);
      continue;
    }
    if (!ensure_host_steps(c, 1024) || (c->steps.n < (size_t)1024 && c->steps.alloc(1024))) {
      c->last_error = ONTC_CUDA_FAILURE;
      out[i] = make_progress(ONTC_TRAIN_ERROR, ONTC_CUDA_FAILURE, c);
      continue;
    }
    active[i] = 1;
  }
  // BF16 contexts (at most kMaxTileMats of each profile shape) share their tile launches: one
  // per shape and step, its SMs split among the materials
  std::vector<int> shape_of(n, -1);
  std::vector<std::array<int, 3>> shapes;
  std::vector<int> per_shape;
  bool shared = true;
  int n_active = 0;
  for (int i = 0; i < n; i++) {
    if (!active[i]) continue;
    n_active++;
    const ontc_context* c = ctxs[i];
    if (c->precision != ONTC_PRECISION_BF16) shared = false;
    const std::array<int, 3> key = {c->C0, c->C1, c->model().Fp};
    int sh = 0;
    while (sh < (int)shapes.size() && shapes[sh] != key) sh++;
    if (sh == (int)shapes.size()) {
      shapes.push_back(key);
      per_shape.push_back(0);
    }
    shape_of[i] = sh;
    if (++per_shape[sh] > kMaxTileMats) shared = false;
  }
  if (shared && n_active >= 2) {
    train_shared(ctxs, target, active, shape_of, (int)shapes.size(), err);
  }
  // otherwise one chunk per context in turn: while the host waits for one context's previous
  // chunk, the others' kernels run on their own streams
  for (bool more = !(shared && n_active >= 2); more;) {
    more = false;
    for (int i = 0; i < n; i++) {
      ontc_context* c = ctxs[i];
      if (!active[i] || err[i] != cudaSuccess || c->batch_i >= target[i]) continue;
      err[i] = enqueue_chunk(c, target[i]);
      more = true;
    }
  }
  int result = ONTC_SUCCESS;
  for (int i = 0; i < n; i++) {
    if (active[i]) finish_train(ctxs[i], err[i], &out[i]);
    if (result == ONTC_SUCCESS && out[i].result != ONTC_SUCCESS) result = out[i].result;
  }
  return result;
}

void ontc_eval(ontc_context* c, ontc_eval_results* out)
{
  *out = ontc_eval_results{};
  if (!c->manifest_loaded || (c->train_phase != ONTC_TRAIN_IN_PROGRESS && c->train_phase != ONTC_TRAIN_COMPLETE)) {
    c->last_error = ONTC_INVALID_STATE;
    return;
  }
  std::vector<double> sums;
  if (full_forward(c, kEval, &sums) != cudaSuccess) {
    c->last_error = ONTC_CUDA_FAILURE;
    return;
  }
  double num = 0.0, den = 0.0;
  for (int m = 0; m < c->mips; m++) {
    num += sums[m];
    den += (double)c->mip_dim[m] * c->mip_dim[m] * c->C;
  }
  out->mse = num / den;
  out->psnr = -10.0 * std::log10(out->mse);
}

int ontc_decoder_create_float(ontc_context* c, int32_t mode, void* stream, ontc_decoder** out)
{
  if (!out) return ONTC_INVALID_STATE;
  *out = nullptr;
  if (!c || !c->manifest_loaded || c->train_phase != ONTC_TRAIN_COMPLETE) return ONTC_INVALID_STATE;
  if (mode != ONTC_DECODE_FP32 && mode != ONTC_DECODE_BF16 && mode != ONTC_DECODE_FP8) return ONTC_INVALID_STATE;
  ontc_compressed_data cd;
  ontc_get_compressed_data(c, &cd);
  int r = ontc_decoder_create(&cd, ONTC_DECODE_INT8, stream, out);
  if (r != ONTC_SUCCESS) return r;
  std::vector<float> W(c->nW);
  if (cudaMemcpy(W.data(), c->W.p, c->nW * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    r = ONTC_CUDA_FAILURE;
  if (r == ONTC_SUCCESS) r = ontc::decoder_set_float(*out, mode, W.data(), c->F, c->C, c->caldata);
  if (r != ONTC_SUCCESS) {
    ontc_decoder_destroy(*out);
    *out = nullptr;
  }
  return r;
}

void ontc_eval_decoded(ontc_context* c, ontc_eval_results* out)
{
  *out = ontc_eval_results{};
  if (!c->manifest_loaded || c->train_phase != ONTC_TRAIN_COMPLETE) {
    c->last_error = ONTC_INVALID_STATE;
    return;
  }
  double num = 0.0;
  if (decoded_sq_err_all(c, &num) != cudaSuccess) {
    c->last_error = ONTC_CUDA_FAILURE;
    return;
  }
  double den = 0.0;
  for (int m = 0; m < c->mips; m++) den += (double)c->mip_dim[m] * c->mip_dim[m] * c->C;
  out->mse = num / den;
  out->psnr = -10.0 * std::log10(out->mse);
}

void ontc_calibrate(ontc_context* c, float headroom, ontc_calibration* out)
{
  *out = ontc_calibration{};
  if (!c->manifest_loaded || c->train_phase != ONTC_TRAIN_COMPLETE) {
    c->last_error = ONTC_INVALID_STATE;
    return;
  }
  cudaError_t e;
  *out = calibrate(c, headroom, &e);
  if (e != cudaSuccess) {
    c->last_error = ONTC_CUDA_FAILURE;
    *out = ontc_calibration{};
  }
}

void ontc_get_compressed_data(ontc_context* c, ontc_compressed_data* d)
{
  memset(d, 0, sizeof(*d));
  if (!c->manifest_loaded) return;
  for (int i = 0; i < c->levels; i++) {
    d->g0[i] = c->g0_host[i];
    d->g0_size[i] = c->level_elems(0, i) * c->b0 / 8;
    d->g1[i] = c->g1_host[i];
    d->g1_size[i] = c->level_elems(1, i) * c->b1 / 8;
  }
  for (int i = 1; i < c->levels; i++) {
    d->g0_offset[i] = d->g0_offset[i - 1] + d->g0_size[i - 1];
    d->g1_offset[i] = d->g1_offset[i - 1] + d->g1_size[i - 1];
  }
  d->g0_total_size = d->g0_offset[c->levels - 1] + d->g0_size[c->levels - 1];
  d->g1_total_size = d->g1_offset[c->levels - 1] + d->g1_size[c->levels - 1];
  d->decoder = c->decoder_host.data();
  d->decoder_size = c->decoder_host.size();
  for (int i = 0; i < c->levels; i++) {
    d->g0_grid_dim[i] = c->g0_dim[i];
    d->g1_grid_dim[i] = c->g1_dim[i];
  }
  d->profile = c->profile;
  d->g0_bits_per_channel = c->b0;
  d->g1_bits_per_channel = c->b1;
  d->g0_channels = c->C0;
  d->g1_channels = c->C1;
  d->dim = c->mip_dim[0];
  d->mip_count = c->mips;
  d->level_count = c->levels;
  d->caldata = c->caldata;
  d->channel_count = 0;
  for (int i = 0; i < c->source_count; i++)
    for (int k = 0; k < c->sources[i].nch && d->channel_count < ONTC_MAX_CHANNELS; k++)
      d->channel_semantics[d->channel_count++] = c->sources[i].sem;
}

void ontc_get_texture_data(ontc_context* c, ontc_texture_data* t)
{
  memset(t, 0, sizeof(*t));
  if (!c->manifest_loaded) return;
  t->tex_count = c->source_count;
  t->mip_count = c->mips;
  for (int i = 0; i < c->source_count; i++) {
    t->semantics[i] = c->sources[i].sem;
    t->channels[i] = c->sources[i].nch;
    for (int m = 0; m < c->mips; m++) t->mips[i][m] = c->mips_host[i][m].empty() ? nullptr : c->mips_host[i][m].data();
  }
}

int32_t ontc_get_mip_dim(ontc_context* c, int32_t mip)
{
  if (c->initialized && c->manifest_loaded && mip >= 0 && mip < c->mips) return c->mip_dim[mip];
  return 0;
}

int32_t ontc_feature_level_for_lod(ontc_context* c, int32_t lod) { return c->feature_level_for_lod(lod); }

int ontc_get_last_error(ontc_context* c) { return c->last_error; }

int32_t ontc_steps_for_quality(int32_t q)
{
  switch (q) {  // libopenntc.cpp:428-443
    case ONTC_QUALITY_LOW: return 30000;
    case ONTC_QUALITY_MEDIUM: return 120000;
    case ONTC_QUALITY_HIGH: return 240000;
    case ONTC_QUALITY_ULTRA: return 480000;
    default: return 30000;
  }
}

int ontc_get_step_losses(ontc_context* c, double* out, int32_t n)
{
  if (!c->manifest_loaded || !c->losses.p || n <= 0) return ONTC_INVALID_STATE;
  n = std::min(n, c->batch_i);
  if (n == 0) return ONTC_SUCCESS;
  if (cudaMemcpy(out, c->losses.p + (c->batch_i - n), n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return ONTC_CUDA_FAILURE;
  return ONTC_SUCCESS;
}

int64_t ontc_kernel_launch_count(ontc_context* c) { return c->launches; }

int64_t ontc_texels_trained(ontc_context* c) { return c->texels_trained; }

int ontc_profile_kernels(ontc_context* c, int32_t enable)
{
  if (!c->initialized) return ONTC_INVALID_STATE;
  cudaStreamSynchronize(c->stream);
  for (auto& r : c->prof) {
    c->event_pool.push_back(r.a);
    c->event_pool.push_back(r.b);
  }
  c->prof.clear();
  c->profiling = enable != 0;
  return ONTC_SUCCESS;
}

int ontc_kernel_times(ontc_context* c, ontc_kernel_time* out, int32_t max_classes)
{
  if (!c->initialized || !out) return 0;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return 0;
  int n = std::min<int>(max_classes, ONTC_KCLASS_COUNT);
  for (int i = 0; i < n; i++) out[i] = ontc_kernel_time{};
  for (auto& r : c->prof) {
    if (r.cls >= n) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    out[r.cls].launches += 1;
    out[r.cls].total_ms += ms;
    out[r.cls].bytes += r.bytes;
    out[r.cls].flops += r.flops;
  }
  return n;
}

const char* ontc_version(void) { return "ontc 0.1 sm_100a"; }

}  // extern "C"

// ---- introspection (include/ontc_debug.h) ------------------------------------------------

extern "C" {

int64_t ontc_debug_tensor(ontc_context* c, int32_t which, int32_t level, float* host, int64_t n, int32_t to_device)
{
  float* dev = nullptr;
  size_t count = 0;
  if (which >= ONTC_DBG_G0 && which <= ONTC_DBG_G1_GRAD) {
    if (!c->manifest_loaded || level < 0 || level >= c->levels) return -1;
    static const int map_g[8] = {0, 1, 0, 0, 1, 1, 0, 1};
    static const int map_k[8] = {0, 0, 1, 2, 1, 2, 3, 3};
    const int g = map_g[which], k = map_k[which];
    dev = c->lat[g][k][level].p;
    count = c->level_elems(g, level);
  } else if (which == ONTC_DBG_NOISE0 || which == ONTC_DBG_NOISE1) {
    const int g = which - ONTC_DBG_NOISE0;
    dev = c->noise_buf[g].p;
    count = c->noise_buf[g].n;
    if (!dev) return -1;
  } else if (which == ONTC_DBG_W || which == ONTC_DBG_W_M || which == ONTC_DBG_W_V) {
    if (!c->initialized) return -1;
    dev = which == ONTC_DBG_W ? c->W.p : which == ONTC_DBG_W_M ? c->Wm.p : c->Wv.p;
    count = (size_t)c->nW;
  } else if (which == ONTC_DBG_W_GRAD) {
    if (to_device || c->last_dW.empty()) return -1;
    if (n <= 0) return (int64_t)c->last_dW.size();
    if ((size_t)n > c->last_dW.size()) return -1;
    memcpy(host, c->last_dW.data(), n * sizeof(float));
    return n;
  } else {
    return -1;
  }
  if (n <= 0) return (int64_t)count;
  if ((size_t)n > count || !dev) return -1;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!e)
    e = to_device ? cudaMemcpy(dev, host, n * sizeof(float), cudaMemcpyHostToDevice)
                  : cudaMemcpy(host, dev, n * sizeof(float), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? n : -1;
}

int ontc_debug_last_step(ontc_context* c, ontc_debug_step* o)
{
  memset(o, 0, sizeof(*o));
  const StepRec& s = c->last_step;
  o->lod = s.lod;
  o->n_grids = s.n_grids;
  for (int i = 0; i < kMaxGrids; i++) {
    o->ox[i] = s.ox[i];
    o->oy[i] = s.oy[i];
  }
  o->noise = s.noise;
  o->seed = s.seed;
  o->step = s.step;
  o->level = s.level;
  o->lr_grid = s.lr_grid;
  o->lr_dec = s.lr_dec;
  o->b1 = s.b1;
  o->b2 = s.b2;
  o->gb1 = s.gb1;
  o->gb2 = s.gb2;
  o->grid_update = s.grid_update;
  return ONTC_SUCCESS;
}

int ontc_debug_tile_costs(ontc_context* c, float* out_us, int32_t n)
{
  if (!c->manifest_loaded || !out_us || n < c->mips) return ONTC_INVALID_STATE;
  if (tune_tiles(c) != cudaSuccess) return ONTC_CUDA_FAILURE;
  for (int l = 0; l < n; l++) out_us[l] = l < c->mips ? c->unit_us[l] : 0.0f;
  return ONTC_SUCCESS;
}

int ontc_debug_gradients(ontc_context* c, ontc_debug_step* d, double* loss)
{
  if (!c->manifest_loaded || d->lod < 0 || d->lod >= c->mips || d->n_grids < 1 || d->n_grids > kMaxGrids)
    return ONTC_INVALID_STATE;
  StepRec s = {};
  s.lod = d->lod;
  s.level = c->feature_level_for_lod(d->lod);
  d->level = s.level;
  s.mip_dim = c->mip_dim[d->lod];
  s.tile_dim = std::min(s.mip_dim, 256);
  s.n_grids = d->n_grids;
  s.texels = s.n_grids * s.tile_dim * s.tile_dim;
  s.noise = d->noise ? 1 : 0;
  s.grid_update = 1;
  s.seed = d->seed;
  s.norm_lod = d->lod / static_cast<float>(c->mips - 1);
  s.step = d->step;
  for (int i = 0; i < kMaxGrids; i++) {
    s.ox[i] = ((d->ox[i] % s.mip_dim) + s.mip_dim) % s.mip_dim;
    s.oy[i] = ((d->oy[i] % s.mip_dim) + s.mip_dim) % s.mip_dim;
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  for (int g = 0; g < 2 && !e; g++)
    e = cudaMemsetAsync(c->lat[g][3][s.level].p, 0, c->level_elems(g, s.level) * sizeof(float), c->stream);
  if (!e) e = cudaMemcpyAsync(c->aux_steps.p, &s, sizeof(s), cudaMemcpyHostToDevice, c->stream);
  const int units = (s.texels + kTile - 1) / kTile;
  int grid = std::min(units, c->sms);
  const Model M = c->model();
  TileOut to = {c->dWpart.p, c->loss_part.p, nullptr};
  bool acc = false;  // the tcgen05 tile kernels accumulate into row 0 (zero before and after)
  if (!e) e = cudaMemsetAsync(c->dWpart.p, 0, c->nW * sizeof(float), c->stream);
  if (!e) {
    if (c->precision == ONTC_PRECISION_BF16 || c->precision == ONTC_PRECISION_BF16X3) {
      acc = true;
      const bool split = c->precision == ONTC_PRECISION_BF16X3;
      const int gpc = tc_groups_per_cta(split);
      grid = std::min((units + gpc - 1) / gpc, tc_max_grid());
      e = launch_tc_units(M, c->aux_steps.p, 0, grid, to, c->tc_error.p, c->boxes[s.lod], split, c->stream);
      if (e == cudaErrorNotSupported) {
        cudaGetLastError();
        acc = false;
        grid = std::min(units, c->sms);
        e = launch_simt_units(kTrain, M, c->aux_steps.p, 0, grid, to, c->stream);
      }
    } else {
      e = launch_simt_units(kTrain, M, c->aux_steps.p, 0, grid, to, c->stream);
    }
    c->launches++;
  }
  const int rows = acc ? 1 : grid;
  std::vector<float> part((size_t)rows * c->nW);
  std::vector<double> lp(grid);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (!e && tc_failed(c)) e = cudaErrorLaunchTimeout;
  if (!e) e = cudaMemcpy(part.data(), c->dWpart.p, part.size() * sizeof(float), cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(lp.data(), c->loss_part.p, lp.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemset(c->dWpart.p, 0, c->nW * sizeof(float));
  if (e) return ONTC_CUDA_FAILURE;
  c->last_dW.assign(c->nW, 0.0f);
  for (int w = 0; w < c->nW; w++) {
    double sum = 0.0;
    for (int i = 0; i < rows; i++) sum += part[(size_t)i * c->nW + w];
    c->last_dW[w] = (float)sum;
  }
  double l = 0.0;
  for (double v : lp) l += v;
  if (loss) *loss = l / ((double)c->C * s.texels);
  return ONTC_SUCCESS;
}

int ontc_debug_quantize_pack(const float* host_in, int64_t n, int32_t bits, uint32_t* host_out)
{
  if (bits <= 0 || bits > 16 || (n * bits) % 32 != 0) return ONTC_INVALID_STATE;
  DBuf<float> in;
  DBuf<uint32_t> out;
  const size_t words = (size_t)(n * bits / 32);
  if (in.alloc(n) || out.alloc(words)) return ONTC_ALLOCATION_FAILURE;
  cudaError_t e = cudaMemcpy(in.p, host_in, n * sizeof(float), cudaMemcpyHostToDevice);
  if (!e) e = launch_quantize_pack(in.p, n, bits, out.p, 0);
  if (!e) e = cudaMemcpy(host_out, out.p, words * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  return e ? ONTC_CUDA_FAILURE : ONTC_SUCCESS;
}

int ontc_debug_lanczos_down(const uint8_t* src, int32_t dim, int32_t ch, uint8_t* dst)
{
  DBuf<uint8_t> s, d;
  DBuf<float> tmp;
  const size_t n = (size_t)dim * dim * ch;
  if (s.alloc(n) || d.alloc(n / 4) || tmp.alloc(n / 2)) return ONTC_ALLOCATION_FAILURE;
  cudaError_t e = cudaMemcpy(s.p, src, n, cudaMemcpyHostToDevice);
  if (!e) e = launch_lanczos_down(s.p, dim, ch, tmp.p, d.p, 0);
  if (!e) e = cudaMemcpy(dst, d.p, n / 4, cudaMemcpyDeviceToHost);
  return e ? ONTC_CUDA_FAILURE : ONTC_SUCCESS;
}

int ontc_debug_lanczos_weights(float* out12) { return lanczos_weights(out12) ? ONTC_CUDA_FAILURE : ONTC_SUCCESS; }

int ontc_debug_package(ontc_context* c, int32_t mip, uint8_t* out)
{
  if (!c->manifest_loaded || mip < 0 || mip >= c->mips) return ONTC_INVALID_STATE;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!e) e = cudaMemcpy(out, c->package[mip].p, c->package[mip].n, cudaMemcpyDeviceToHost);
  return e ? ONTC_CUDA_FAILURE : ONTC_SUCCESS;
}

int64_t ontc_debug_fail_device_alloc(int64_t n)
{
  const int64_t done = g_dev_allocs.load();
  g_fail_alloc.store(n > 0 ? done + n : 0);
  return done;
}

int ontc_debug_exact_gradients(ontc_context* c, int32_t enable)
{
  if (!c) return ONTC_INVALID_STATE;
  c->exact_grad = enable != 0;
  return ONTC_SUCCESS;
}

int ontc_debug_complete(ontc_context* c, const float* s_a)
{
  if (!c || !c->manifest_loaded ||
      (c->train_phase != ONTC_TRAIN_IN_PROGRESS && c->train_phase != ONTC_TRAIN_COMPLETE))
    return ONTC_INVALID_STATE;
  cudaError_t e = drain_side(c);
  if (!e) e = flush_latents(c);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (e) return ONTC_CUDA_FAILURE;
  c->batch_i = c->batch_count;
  c->train_phase = ONTC_TRAIN_COMPLETE;
  e = complete_training(c);
  if (!e && s_a) {
    std::vector<float> Wh(c->nW);
    e = cudaMemcpy(Wh.data(), c->W.p, c->nW * sizeof(float), cudaMemcpyDeviceToHost);
    if (!e) {
      c->caldata.s_a1 = s_a[0];
      c->caldata.s_a2 = s_a[1];
      build_blob(c, Wh, s_a[0], s_a[1], false, c->decoder_host.data());
    }
  }
  return e ? ONTC_CUDA_FAILURE : ONTC_SUCCESS;
}

int ontc_debug_wait_timeout(int32_t polls)
{
  if (polls < 1 || polls > 1000) return ONTC_INVALID_STATE;
  DBuf<int> flag;
  if (flag.alloc(1)) return ONTC_ALLOCATION_FAILURE;
  int h = -1;
  cudaError_t e = launch_wait_check((uint32_t)polls, flag.p, 0);
  if (!e) e = cudaMemcpy(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e) return ONTC_CUDA_FAILURE;
  return h == 1 ? ONTC_CUDA_FAILURE : ONTC_INVALID_STATE;  // the wait must have given up
}

int ontc_debug_cover_op(const int32_t* a, int32_t na, const int32_t* b, int32_t nb, int32_t op, int32_t* out,
                        int32_t cap)
{
  if (op != kCoverInter && op != kCoverMinus) return -1;
  return cover_op(reinterpret_cast<const int (*)[4]>(a), na, reinterpret_cast<const int (*)[4]>(b), nb, op,
                  reinterpret_cast<int (*)[4]>(out), cap);
}

int ontc_debug_disjoint_cover(const int32_t* in, int32_t n, int32_t* out, int32_t cap)
{
  if (n < 0 || cap < 0 || (n > 0 && (!in || !out))) return -1;
  return disjoint_cover(reinterpret_cast<const int (*)[4]>(in), n, reinterpret_cast<int (*)[4]>(out), cap);
}

int ontc_debug_shape(ontc_context* c, int32_t* o)
{
  o[0] = c->F;
  o[1] = c->Fp;
  o[2] = c->C;
  o[3] = c->mips;
  o[4] = c->levels;
  o[5] = c->nW;
  for (int i = 0; i < 6; i++) o[6 + i] = i < c->levels ? c->g0_dim[i] : 0;
  for (int i = 0; i < 6; i++) o[12 + i] = i < c->levels ? c->g1_dim[i] : 0;
  for (int i = 0; i < 12; i++) o[18 + i] = i < c->mips ? c->mip_dim[i] : 0;
  o[30] = c->batch_i;
  o[31] = c->lock_i;
  o[32] = c->batch_count;
  return ONTC_SUCCESS;
}

}  // extern "C"
