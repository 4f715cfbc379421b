/*
 * state.h -- per-handle state that the B200 library adds behind
 * Hcblaslibrary::impl (math mode, device workspace, tuned configurations,
 * diagnostics).  Internal header.
 */
#ifndef HCBLAS_B200_STATE_H_
#define HCBLAS_B200_STATE_H_

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

/* library version: hcblasGetVersionString, and part of every autotune key */
#define HCBLAS_B200_VERSION "0.2.0"

/* one timed kernel launch (events recorded on the launch stream) */
struct HcblasProfRec {
  const char *name;
  void *ev0; /* cudaEvent_t */
  void *ev1;
};

/* The last grouped-GEMM plan of a handle: the device problem table (entries
 * then tile prefix sums), its pinned host staging copy, and the key that lets
 * an identical follow-up call skip the tensor-map encoding and the upload. */
struct HcblasGroupedPlan {
  void *table = nullptr; /* device */
  size_t table_bytes = 0;
  int table_device = -1;
  void *staging = nullptr; /* pinned host */
  size_t staging_bytes = 0;
  void *upload_done = nullptr; /* cudaEvent_t recorded after the staging copy */
  std::vector<unsigned char> key;
  std::vector<unsigned char> compact_key; /* strided batches: a short key equivalent to `key` */
  int count = 0;       /* problems in the device table */
  int total_tiles = 0;
  size_t tile_start_offset = 0;
  size_t tile_desc_offset = 0; /* per-tile descriptors (hcbk_grouped_fill_tiles) */
  std::vector<int> fallback; /* problems the table cannot hold (TMA alignment) */
  int64_t work = 0;          /* padded tensor work of the table (bucket of the tuner) */
  int tuned_ctas = 0;        /* CTAs per SM chosen by the autotuner; 0 = not tuned */
  /* split-BF16 SGEMM plans only: the bf16 planes of every problem (device),
   * and the pack jobs' place in the table */
  void *planes = nullptr;
  size_t planes_bytes = 0;
  int pack_count = 0;
  int pack_tiles = 0;
  size_t pack_offset = 0;
  size_t pack_ts_offset = 0;
};

/* One captured call sequence (hcblasSetTuningParam "graphs"): the key is the
 * canonical call, the knobs that steer dispatch, the stream and the
 * workspace generation; `launches` is the number of kernels it replays. */
struct HcblasGraphEntry {
  std::vector<unsigned char> key;
  void *exec = nullptr; /* cudaGraphExec_t */
  long long launches = 0;
  const char *path = "";
};

struct HcblasB200State {
  int math_mode = 0;   /* HCBLAS_MATH_* */
  int math_param = 0;  /* terms (split-BF16) or slices (Ozaki) */
  int split_promote_kb = 1; /* split-BF16: K-slabs per TMEM chunk (tuning knob) */
  int tc_pair = 1; /* CTA-pair (cta_group::2) tensor-core kernels: 0 never, 1 auto, 2 always */
  int crt_i8 = 1;  /* CRT DGEMM modular GEMMs: 1 int8 residues on kind::i8, 0 binary16 */
  int grouped_ctas = 2; /* grouped f16 kernel: CTAs per SM (1: 6-stage ring, 2: 3 stages each) */
  int grouped_c_tma = 1; /* grouped f16 kernel: C through TMA boxes where C allows (0: stores) */
  int dgemm_dmma = 1; /* native D/Z GEMM: 1 FP64 tensor path (mma.sync .f64), 0 CUDA-core FMA */
  int ozaki_default_slices = 7; /* Ozaki slices when the mode's param is 0 */
  /* requested accuracy of the emulated modes in bits (hcblasSetAccuracyTarget;
   * 0: each mode's default count, -1: the format's native precision) */
  int accuracy_bits = 0;
  const char *last_path = "none";
  /* device workspace owned by the handle (grown on demand, freed at destroy) */
  void *workspace = nullptr; /* cudaMallocAsync'd, released stream-ordered */
  size_t workspace_bytes = 0;
  int workspace_device = -1;
  void *workspace_stream = nullptr; /* stream of the last call that used it */
  void *workspace_event = nullptr;  /* cudaEvent_t ordering a new stream after it */
  size_t workspace_limit = 0;       /* tuning knob "workspace_mb" (0 = none) */
  /* device error block of the tensor-core kernels: int 0 is set when a
   * pipeline wait times out, ints 2-3 hold the wait limit in ns */
  int *dev_err = nullptr;
  int dev_err_device = -1;
  unsigned long long wait_limit_ns = 0; /* tuning knob "wait_timeout_us" (0 = 2 s) */
  int inject_timeout = 0; /* tuning knob "inject_timeout": arms the next HGEMM call */
  /* a second stream of the handle's device for independent passes within one
   * call (forked from and joined back into the call's stream by events);
   * tuning knob "aux_stream" (1 = use it) */
  int use_aux = 1;
  void *aux_stream = nullptr;
  int aux_device = -1;
  void *aux_fork = nullptr, *aux_join = nullptr;
  /* per-kernel CUDA-event timing (hcblasSetProfiling) */
  bool profiling = false;
  std::vector<HcblasProfRec> prof;
  std::vector<void *> event_pool;
  HcblasGroupedPlan grouped;
  HcblasGroupedPlan grouped_split; /* hcblasSgemmGrouped (split-BF16) */
  HcblasGroupedPlan grouped_simt;  /* hcblas{D,C,Z}gemmGrouped (CUDA cores) */
  HcblasGroupedPlan grouped_ptr;   /* pointer-array HGEMM batches (device-built table) */
  /* CUDA-graph replay of repeated identical calls (off by default) */
  int graphs = 0;
  /* time candidate tile configurations per size bucket (off by default) */
  int autotune = 0;
  unsigned workspace_epoch = 0; /* bumped whenever a buffer a graph may reference moves */
  std::vector<HcblasGraphEntry> graph_cache;
};

namespace hcblas_b200 {

/* cumulative number of kernels launched by this library in this process */
void count_launch(int n = 1);
long long launch_count();
void *prof_event(HcblasB200State *st);
void prof_record(void *ev, void *stream);

/* Fork the handle's second stream off `stream` (it waits for everything
 * queued on `stream` so far) and return it, or nullptr when the knob is off
 * or the stream cannot be had (the caller then stays on `stream`). */
void *aux_fork(HcblasB200State *st, void *stream);
/* Make `stream` wait for everything queued on the second stream. */
int aux_join(HcblasB200State *st, void *stream);

/* Run `fn` (one library call, returning an HCBK_* code, that launches
 * `kernels` kernels); when profiling is on, bracket it with CUDA events on
 * `stream`.  Counts every kernel launch. */
template <typename F>
int timed_launch(HcblasB200State *st, void *stream, const char *name, F &&fn, int kernels = 1) {
  if (st && st->profiling) {
    void *e0 = prof_event(st);
    void *e1 = prof_event(st);
    prof_record(e0, stream);
    int rc = fn();
    prof_record(e1, stream);
    st->prof.push_back(HcblasProfRec{name, e0, e1});
    if (rc == 0) count_launch(kernels);
    return rc;
  }
  int rc = fn();
  if (rc == 0) count_launch(kernels);
  return rc;
}

/* Make `dev` current for the lifetime of the guard, restoring the previous
 * device afterwards. */
class DeviceGuard {
 public:
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
  bool ok() const { return ok_; }

 private:
  int prev_ = -1;
  bool ok_ = false;
};

/* The handle's workspace of at least `bytes` on the current device, for
 * work enqueued on `stream`: the stream is ordered after the workspace's
 * last use on another stream; growth releases the old buffer and allocates
 * the new one stream-ordered (cudaFreeAsync / cudaMallocAsync), so no
 * device-wide wait is made.  nullptr when the workspace must grow while
 * `stream` is being captured, beyond the "workspace_mb" limit, or when the
 * allocation fails. */
void *ensure_workspace(HcblasB200State *st, size_t bytes, void *stream);

/* The handle's device error flag on the current device (allocated and
 * zeroed on first use); nullptr if it cannot be allocated. */
int *device_error_flag(HcblasB200State *st);

/* Destroy every cached graph (their buffers moved or the handle dies). */
void clear_graph_cache(HcblasB200State *st);

/* HCBLAS_LOG=1 prints one line per GEMM call with the path taken. */
bool log_enabled();

}  // namespace hcblas_b200

#endif /* HCBLAS_B200_STATE_H_ */
