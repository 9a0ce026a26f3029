// Internal definitions shared by the libamk translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "amk.h"
#include "morton.cuh"

namespace amk {

// ---------------------------------------------------------------- constants
// utils/constants.h:11-38 of the reference.
constexpr double kPi = 3.14159265358979323846;
constexpr double kElementaryCharge = 1.602176634e-19;
constexpr double kElectronMass = 9.1093837015e-31;
constexpr double kProtonMass = 1.67262192369e-27;
constexpr double kNeutronMass = 1.67492749804e-27;
constexpr double kCoulombConstant = 8.9875517923e9;
constexpr double kBoltzmann = 1.380649e-23;
constexpr double kSpeedOfLight = 2.99792458e8;
// Pairs closer than this (m^2) are skipped: coulomb_interaction.cc:19,
// barnes-hut.cc:17, fast-multipole.cc:259.
constexpr double kMinSquaredDistance = 1e-30;

// ---------------------------------------------------------------- errors
void set_error(int code, const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define AMK_CUDA_TRY(expr)                                                       \
  do {                                                                          \
    cudaError_t amk_err_ = (expr);                                              \
    if (amk_err_ != cudaSuccess)                                                \
      return ::amk::fail(AMK_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,           \
                         cudaGetErrorString(amk_err_), __FILE__, __LINE__);     \
  } while (0)

#define AMK_TRY(expr)              \
  do {                             \
    int amk_rc_ = (expr);          \
    if (amk_rc_ != AMK_OK) return amk_rc_; \
  } while (0)

// ---------------------------------------------------------------- buffers
// A growable device allocation. Growth reallocates without preserving the
// contents; callers that need the contents use reserve_keep().
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  int reserve(size_t want) {
    if (want <= bytes) return AMK_OK;
    release();
    size_t b = want + want / 4 + 256;
    if (cudaMalloc(&ptr, b) != cudaSuccess) {
      cudaGetLastError();
      ptr = nullptr;
      return fail(AMK_ERR_NOMEM, "device allocation of %zu bytes failed", b);
    }
    bytes = b;
    return AMK_OK;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
  void swap(DevBuf& o) {
    std::swap(ptr, o.ptr);
    std::swap(bytes, o.bytes);
  }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// ---------------------------------------------------------------- particle views
// Structure-of-arrays particle set on the device. Positions are FP64 and
// trap-centred. `q_e` is the charge in units of e (float, exact for +-e) and
// `hq`/`lo` are the double-float split of the scaled position used by the
// FP32 pair kernels: x / L = hq.x + lo.x (|lo| <= ulp(hq)/2), hq.w = q_e
// (0 for dead or neutral particles so that they drop out of every sum).
struct View {
  long n = 0;
  double* x = nullptr;
  double* y = nullptr;
  double* z = nullptr;
  double* q = nullptr;      // charge [C]
  uint8_t* alive = nullptr; // may be null = all alive
  float4* hq = nullptr;
  float4* lo = nullptr;
  double* fx = nullptr;     // force outputs [N]
  double* fy = nullptr;
  double* fz = nullptr;
  double* phi = nullptr;    // optional potential output sum q_j/r (no k)
  double length_scale = 1.0;  // L, a power of two
};

// ---------------------------------------------------------------- context
struct Scratch {
  DevBuf b[128];
};

enum ScratchSlot {
  kSlotPartial = 0,
  kSlotKeysA,
  kSlotKeysB,
  kSlotValsA,
  kSlotValsB,
  kSlotSortHist,
  kSlotSortFlags,
  kSlotCellStart,
  kSlotReduce,
  kSlotTreeKeys,
  kSlotTreeNodesF,
  kSlotTreeNodesI,
  kSlotTreeAux0,
  kSlotTreeAux1,
  kSlotTreeAux2,
  kSlotTreeAux3,
  kSlotTreeAux4,
  kSlotTreeAux5,
  kSlotSorted0,
  kSlotSorted1,
  kSlotSorted2,
  kSlotFmmM,
  kSlotFmmL,
  kSlotFmmLists0,
  kSlotFmmLists1,
  kSlotFmmLists2,
  kSlotFmmLists3,
  kSlotFmmAux0,
  kSlotFmmAux1,
  kSlotFmmAux2,
  kSlotAnnEdges,
  kSlotAnnAux,
  kSlotAnnBest,
  kSlotStatus,
  kSlotMlp0,
  kSlotMlp1,
  kSlotMlp2,
  kSlotMlp3,
  kSlotMlp4,
  kSlotMlp5,
  kSlotAuxState0,
  kSlotAuxState1,
  kSlotAuxState2,
  kSlotAuxState3,
  kSlotAuxState4,
  kSlotAuxState5,
  kSlotAuxState6,
  kSlotScanSums,
  kSlotTreeFrame,
  kSlotTreeL,
  kSlotTreeLeafDepth,
  kSlotTreeCount,
  kSlotTreeBase,
  kSlotTreeCenter,
  kSlotTreeChild,
  kSlotTreeRange,
  kSlotTreeMeta,
  kSlotTreeParent,
  kSlotTreeSrc,
  kSlotTreeOrder,
  kSlotTreeSortedKeys,
  kSlotBhPos,
  kSlotBhNeg,
  kSlotWalkOut,
  kSlotFmmRadius,
  kSlotFmmWork0,
  kSlotFmmWork1,
  kSlotFmmWork2,
  kSlotFmmWork3,
  kSlotFmmWork4,
  kSlotFmmWork5,
  kSlotP2PWork,
  kSlotP2PPart,
  kSlotP2PStage,
  kSlotM2lCodes,
  kSlotM2lTarget,
  kSlotM2lHist,
  kSlotM2lStart,
  kSlotM2lUsed,
  kSlotM2lClassIndex,
  kSlotM2lTiles,
  kSlotM2lTileStart,
  kSlotM2lCounters,
  kSlotM2lPerm,
  kSlotM2lFallback,
  kSlotM2lClassCode,
  kSlotM2lClassEnd,
  kSlotM2lTileClass,
  kSlotM2lTilePos,
  kSlotM2lTable,
  kSlotM2lHash,
  kSlotM2lSplit,
  kSlotM2lUnitDesc,
  kSlotM2lPairSrc,
  kSlotM2lTable3,
  kSlotM2lRefl,
  kSlotFmmNodeRec,
  kNumSlots
};
static_assert(kNumSlots <= 128, "scratch slots");

struct PhaseClock {
  cudaEvent_t start[AMK_NUM_PHASES] = {};
  cudaEvent_t stop[AMK_NUM_PHASES] = {};
  double ms[AMK_NUM_PHASES] = {};
  long launches[AMK_NUM_PHASES] = {};
  bool pending[AMK_NUM_PHASES] = {};
};

struct Fmm;  // fmm.cu
struct Mlp;  // mlp.cu
struct Batch;  // batch.cu

}  // namespace amk

struct amk_ctx {
  amk_params p;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;

  long n = 0;
  long capacity = 0;
  // particle state (device)
  amk::DevBuf x, y, z, vx, vy, vz, fx, fy, fz, q, m, hq, lo, species, alive, ids;
  double length_scale = 1.0;
  bool staggered = false;     // first push done (lorentz.h:34)
  long step = 0;              // completed steps
  bool stage_dirty = true;    // hq/lo must be rebuilt from x,y,z
  // Morton order of the all-pairs kernel, reused for a few calls
  amk::DevBuf ap_perm;
  long ap_perm_n = -1;
  int ap_perm_age = 0;
  // aux particle set for the stateless solver mirrors
  amk::DevBuf ax, ay, az, aq, ahq, alo, afx, afy, afz, aphi;
  long aux_capacity = 0;

  amk::Scratch scratch;
  amk::DevBuf host_status;  // pinned host word for small readbacks (unused)

  // energy time-centring (EnergyHistory, energy_analysis.h:23-28)
  bool energy_has_previous = false;
  double prev_trap = 0.0, prev_coulomb = 0.0;

  bool profiling = false;
  amk::PhaseClock clock;
  long kernel_launches = 0;

  amk::Fmm* fmm = nullptr;
  amk::Mlp* mlp = nullptr;
  amk::Batch* batch = nullptr;  // batched instances over segment offsets
  // leaf capacities of the context's own solver calls (the reference's 32 and
  // 8 unless amk_autotune or amk_set_leaf_sizes changed them)
  int fmm_leaf = 32;
  int fmm_precision = 0;  // AMK_FMM_FP64 or AMK_FMM_TENSOR (M2L class products)
  int bh_leaf = 8;
  // learned FMM correction state
  bool learned_trained = false;
  bool learned_fallback = false;
  double learned_last_error = -1.0;
};

namespace amk {

// Phase timing: wraps one phase in events on the context stream when
// profiling is enabled (events are read lazily in amk_phase_times).
int phase_begin(amk_ctx* c, int phase);
int phase_end(amk_ctx* c, int phase);
// the same, with the events recorded on another stream of the context
int phase_begin_on(amk_ctx* c, int phase, cudaStream_t stream);
int phase_end_on(amk_ctx* c, int phase, cudaStream_t stream);

inline int check_launch(amk_ctx* c, const char* what) {
  c->kernel_launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(AMK_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return AMK_OK;
}

template <typename T>
inline T* slot(amk_ctx* c, int s, size_t count, int* rc) {
  *rc = c->scratch.b[s].reserve(count * sizeof(T));
  return c->scratch.b[s].as<T>();
}

// Species defaults (particle_species.h:27-46).
void species_properties(int s, double* m, double* q);
bool is_antiparticle_pair(int a, int b);

// View over the context's main particle state.
View main_view(amk_ctx* c);

// Rebuilds hq/lo (double-float staging) of a view on the context stream.
int stage_view(amk_ctx* c, const View& v);

// Solvers on a view; outputs into v.fx/fy/fz (and v.phi when non-null).
int allpairs_forces(amk_ctx* c, const View& v);
int cutoff_forces(amk_ctx* c, const View& v, double cutoff, double* energy_out);
int barnes_hut_forces(amk_ctx* c, const View& v, double theta, long leaf_capacity);
int fmm_forces(amk_ctx* c, const View& v, int order, double theta, long leaf_capacity,
               bool learned, double* energy_out);

// Learned correction (mlp.cu / fmm.cu).
int mlp_forward_device(amk_ctx* c, const float* x, long n, float* y);
int mlp_check_status(amk_ctx* c);
int mlp_train_device(amk_ctx* c, const float* x, const float* target, long n, int steps, long batch, float lr,
                     float* final_loss);
int fmm_train_learned(amk_ctx* c, const View& v, double theta, int sample_leaves, int steps, long batch, float lr,
                      float* loss_out, long* samples_out);
int fmm_audit(amk_ctx* c, const View& v, int order, double theta, bool learned, long samples, double* rms);

// Copies host sources into the context's auxiliary set (solver mirrors).
int load_aux_view(amk_ctx* c, long n, const double* x, const double* y, const double* z, const double* q,
                  View* out);

// Power-of-two length scale for a set of host coordinates.
double length_scale_for(double max_abs);

// Radix sort of (key, value) pairs on the context stream: keys 64-bit, values
// 32-bit; sorts `n` elements on bits [0, key_bits); result in keys_out/vals_out.
int radix_sort_pairs(amk_ctx* c, const uint64_t* keys_in, const uint32_t* vals_in,
                     uint64_t* keys_out, uint32_t* vals_out, long n, int key_bits);

// Exclusive prefix sum of int32 values; *total_dev receives the sum.
int exclusive_scan_int(amk_ctx* c, const int* in, long n, int* out, int* total_dev);

// ---------------------------------------------------------------- octree
// The reference's octrees (barnes-hut.cc:38-164, fast-multipole.cc:234-311,
// :342-397) rebuilt from sorted Morton keys. Tree coordinates: Barnes-Hut
// uses physical positions; the FMM rescales to a unit cube,
// x' = (x - mid) / length (fast-multipole.cc:355-390).
constexpr int kTreeLevels = 21;  // 63-bit keys: depth limit 21 (reference: 32)

struct TreeFrame {
  double mid[3];     // FMM: bbox centre (0 for Barnes-Hut)
  double length;     // FMM: cube edge (1 for Barnes-Hut)
  double root_c[3];  // root cube centre in tree coordinates
  double root_h;     // root half edge in tree coordinates
};

struct Octree {
  long m = 0;                  // sources in the tree, sorted positions [0, m)
  long n_nodes = 0;
  int leaf_cap = 8;
  int max_depth = 0;           // deepest node
  TreeFrame* frame = nullptr;  // device
  uint32_t* order = nullptr;   // sorted position -> view index
  uint64_t* keys = nullptr;    // sorted keys
  double4* src = nullptr;      // sorted sources: tree coordinates + charge
  double4* center = nullptr;   // node centre (tree coordinates) + half edge
  int* child = nullptr;        // 8 per node, -1 = none (octant order)
  int2* range = nullptr;       // node particle range [begin, end)
  uchar2* meta = nullptr;      // (depth, is_leaf)
  int* parent = nullptr;       // -1 for the root
};

// mode 0: Barnes-Hut (sources = live particles, physical coordinates);
// mode 1: FMM (sources = live charged particles, unit-cube coordinates).
int build_octree(amk_ctx* c, const View& v, int leaf_cap, int mode, Octree* out);

// Deterministic FP64 sum of `n` doubles into *out_dev (device pointer).
int reduce_sum(amk_ctx* c, const double* in, long n, double* out_dev);

// Per-step behaviours (push.cu, cellist.cu).
int push_step(amk_ctx* c, uint64_t step_index);
int annihilate_step(amk_ctx* c, uint64_t step_index, long* marked);
// Annihilation on a view (indices, species and ids relative to the view).
int annihilate_view(amk_ctx* c, const View& v, const uint8_t* species, const uint32_t* ids, double radius,
                    double probability, uint32_t seed, uint64_t step_index, long* marked);
// Batched instances (batch.cu).
void batch_destroy(amk_ctx* c);
// Coulomb potential energy (J) of a view under an energy method (energy.cu).
int coulomb_energy_view(amk_ctx* c, View v, const amk_params& p, int method, double* out_host);
// RMS / max relative error of a view's forces against the FP64 exact sum
// over `samples` evenly spaced usable particles (audit.cu).
int force_error(amk_ctx* c, const View& v, long samples, double* rms, double* max_rel);
// Median device time (ms) of `reps` calls after one warm call (audit.cu).
int time_solver(amk_ctx* c, const std::function<int()>& call, int reps, double* ms);

}  // namespace amk
