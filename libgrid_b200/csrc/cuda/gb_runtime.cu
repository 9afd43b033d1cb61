// libgrid-b200 CUDA runtime: device selection, the library stream, error
// latch, launch counter, memory helpers, timing events, library-owned device
// scratch and FFT twiddle tables.
//
// Replaces the reference's GPU memory manager for this path (src/cuda.c):
// one GPU, device-resident buffers owned by the host layer, no swap cache,
// no CPU fallback.  Library scratch (twiddles, kinetic tables, reduction
// partials, line-solver coefficients) lives in named slots that grow on
// demand and are released at gb_shutdown.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cudaTypedefs.h>

#include "gb_common.cuh"
#include "gb_internal_cuda.h"

static int g_device = -1;
static cudaStream_t g_stream = nullptr;
static int g_err = 0;
static char g_err_where[160] = "";
static long g_launches = 0;

// Scratch buffers replaced while a captured graph is alive stay allocated
// (the graph may hold their address) until the last graph is freed.
static int g_graphs_live = 0;
static void *g_retired[64];
static int g_nretired = 0;

static void free_retired(void) {
  if (g_nretired) cudaStreamSynchronize(g_stream);
  for (int i = 0; i < g_nretired; i++) cudaFree(g_retired[i]);
  g_nretired = 0;
}

static cudaEvent_t g_events[16];
static bool g_events_made = false;

struct Scratch {
  void *p;
  size_t bytes;
};
static Scratch g_scratch[GB_SCR_COUNT];

struct Twiddle {
  void *d64;
  void *d32;
};
static Twiddle g_tw[13];  // index log2(n), n = 2 .. 4096

// Device status block (see "device status" below).
struct IoBlock {
  double2 result[2];
  int status[GB_STATUS_WORDS];
  int pad[16 - GB_STATUS_WORDS];
};
static IoBlock *g_io = nullptr;       // device
static IoBlock *g_io_host = nullptr;  // pinned mirror
static unsigned g_wait_limit = 0;     // 0: each wait's built-in limit

extern "C" void gb__count_launch(void) { g_launches++; }

extern "C" int gb__set_error(int code, const char *where) {
  if (!g_err) {
    g_err = code ? code : -1;
    snprintf(g_err_where, sizeof(g_err_where), "%s", where ? where : "");
  }
  return g_err;
}

extern "C" cudaStream_t gb__stream(void) { return g_stream; }

extern "C" int gb_init(int device) {
  if (g_stream && device == g_device) return 0;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return gb__set_error((int) e, "cudaSetDevice");
  e = cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return gb__set_error((int) e, "cudaStreamCreate");
  g_device = device;
  if (!g_events_made) {
    for (int i = 0; i < 16; i++) cudaEventCreate(&g_events[i]);
    g_events_made = true;
  }
  return 0;
}

extern "C" int gb_shutdown(void) {
  if (!g_stream) return 0;
  cudaStreamSynchronize(g_stream);
  for (int i = 0; i < GB_SCR_COUNT; i++) {
    if (g_scratch[i].p) cudaFree(g_scratch[i].p);
    g_scratch[i].p = nullptr;
    g_scratch[i].bytes = 0;
  }
  for (int i = 0; i < 13; i++) {
    if (g_tw[i].d64) cudaFree(g_tw[i].d64);
    if (g_tw[i].d32) cudaFree(g_tw[i].d32);
    g_tw[i].d64 = g_tw[i].d32 = nullptr;
  }
  return 0;
}

extern "C" int gb_last_error(void) { return g_err; }
extern "C" const char *gb_last_error_where(void) { return g_err_where; }
extern "C" void gb_clear_error(void) {
  g_err = 0;
  g_err_where[0] = 0;
  if (g_io) {
    cudaStreamSynchronize(g_stream);
    cudaMemset(g_io->status, 0, sizeof(int) * GB_STATUS_WORDS);
  }
}

static int check_status(void);

extern "C" int gb_synchronize(void) {
  cudaError_t e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "cudaStreamSynchronize");
  check_status();
  return g_err;
}

extern "C" void *gb_stream_handle(void) { return (void *) g_stream; }
extern "C" long gb_launch_count(void) { return g_launches; }

// CUDA graphs of library calls: gb_graph_begin starts capturing the library
// stream, so the kernels and copies the following calls issue are recorded
// instead of run; gb_graph_end instantiates them into an executable graph
// that gb_graph_launch replays on the stream (the same kernels with the same
// arguments and pointers).  Calls that read results back to the host must
// not be captured; scratch buffers are best sized by one uncaptured run of
// the same calls first (a capture must not free device memory).
struct GbGraph {
  cudaGraphExec_t exec;
  long kernels;  // launches recorded, added to gb_launch_count per replay
};
static long g_capture_start = 0;

extern "C" int gb_graph_begin(void) {
  if (!g_stream) return gb__set_error(1080, "graph: library not initialised");
  const cudaError_t e = cudaStreamBeginCapture(g_stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return gb__set_error((int) e, "graph: begin capture");
  }
  g_capture_start = g_launches;
  return 0;
}

extern "C" int gb_graph_end(void **out) {
  *out = nullptr;
  cudaGraph_t gr = nullptr;
  const cudaError_t e = cudaStreamEndCapture(g_stream, &gr);
  const long kernels = g_launches - g_capture_start;
  g_launches = g_capture_start;
  if (e != cudaSuccess || !gr) {
    if (gr) cudaGraphDestroy(gr);
    cudaGetLastError();
    return gb__set_error(e != cudaSuccess ? (int) e : 1081, "graph: end capture");
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, gr, 0);
  cudaGraphDestroy(gr);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    return gb__set_error((int) ei, "graph: instantiate");
  }
  GbGraph *g = (GbGraph *) malloc(sizeof(GbGraph));
  if (!g) {
    cudaGraphExecDestroy(ex);
    return gb__set_error(2, "graph: host allocation");
  }
  g->exec = ex;
  g->kernels = kernels;
  g_graphs_live++;
  *out = g;
  return 0;
}

extern "C" int gb_graph_launch(void *h) {
  GbGraph *g = (GbGraph *) h;
  if (!g) return gb__set_error(1082, "graph: null handle");
  const cudaError_t e = cudaGraphLaunch(g->exec, g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "graph: launch");
  g_launches += g->kernels;
  return 0;
}

extern "C" int gb_graph_free(void *h) {
  GbGraph *g = (GbGraph *) h;
  if (g) {
    cudaGraphExecDestroy(g->exec);
    free(g);
    if (--g_graphs_live == 0) free_retired();
  }
  return 0;
}

extern "C" void *gb_device_alloc(size_t bytes) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    gb__set_error((int) e, "cudaMalloc");
    return nullptr;
  }
  return p;
}

extern "C" void gb_device_free(void *p) {
  if (p) {
    cudaStreamSynchronize(g_stream);
    cudaFree(p);
  }
}

extern "C" void *gb_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes ? bytes : 16, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

extern "C" void gb_host_free(void *p) {
  if (p) cudaFreeHost(p);
}

extern "C" int gb_h2d(void *dst, const void *src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "h2d");
  return 0;
}

extern "C" int gb_d2h(void *dst, const void *src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, g_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "d2h");
  return check_status();
}

extern "C" int gb_d2d(void *dst, const void *src, size_t bytes) {
  if (dst == src) return 0;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "d2d");
  return 0;
}

extern "C" int gb_memset(void *dst, int value, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(dst, value, bytes, g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "memset");
  return 0;
}

extern "C" int gb_event_record(int slot) {
  if (slot < 0 || slot >= 16) return gb__set_error(1003, "event slot");
  cudaError_t e = cudaEventRecord(g_events[slot], g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "cudaEventRecord");
  return 0;
}

extern "C" float gb_event_elapsed_ms(int a, int b) {
  float ms = -1.0f;
  if (a < 0 || a >= 16 || b < 0 || b >= 16) return -1.0f;
  cudaEventSynchronize(g_events[b]);
  if (cudaEventElapsedTime(&ms, g_events[a], g_events[b]) != cudaSuccess) {
    cudaGetLastError();
    return -1.0f;
  }
  return ms;
}

void *gb__scratch(int slot, size_t bytes) {
  if (slot < 0 || slot >= GB_SCR_COUNT) return nullptr;
  Scratch &s = g_scratch[slot];
  if (s.bytes >= bytes && s.p) return s.p;
  if (s.p) {
    if (g_graphs_live > 0) {
      // a live graph may hold this buffer's address: keep it until the last
      // graph is freed (a bounded list; beyond it the call fails instead)
      if (g_nretired >= 64) {
        gb__set_error(2, "scratch: too many buffers replaced while CUDA graphs are alive");
        return nullptr;
      }
      g_retired[g_nretired++] = s.p;
    } else {
      cudaStreamSynchronize(g_stream);
      cudaFree(s.p);
    }
  }
  s.p = nullptr;
  s.bytes = 0;
  size_t want = bytes < 4096 ? 4096 : bytes;
  if (cudaMalloc(&s.p, want) != cudaSuccess) {
    cudaGetLastError();
    gb__set_error(2, "scratch cudaMalloc");
    s.p = nullptr;
    return nullptr;
  }
  s.bytes = want;
  return s.p;
}

// ------------------------------------------------------------ pass timing
//
// When enabled, every line pass of the FFT schedules is bracketed by two
// events on the library stream; gb_pass_timing_report sums the elapsed time
// per (program, axis) kind.  Used by the benchmark to time the dominant
// kernel inside the timed region.
#define GB_PASS_SLOTS 8192
static int g_pt_on = 0;
static int g_pt_used = 0;
static cudaEvent_t *g_pt_ev = nullptr;  // 2 per slot
static int *g_pt_kind = nullptr;

extern "C" int gb_pass_timing(int on) {
  if (on && !g_pt_ev) {
    g_pt_ev = (cudaEvent_t *) malloc(sizeof(cudaEvent_t) * 2 * GB_PASS_SLOTS);
    g_pt_kind = (int *) malloc(sizeof(int) * GB_PASS_SLOTS);
    for (int i = 0; i < 2 * GB_PASS_SLOTS; i++) cudaEventCreate(&g_pt_ev[i]);
  }
  g_pt_on = on;
  g_pt_used = 0;
  return 0;
}

int gb__pass_begin(int kind) {
  if (!g_pt_on || g_pt_used >= GB_PASS_SLOTS) return -1;
  const int s = g_pt_used++;
  g_pt_kind[s] = kind;
  cudaEventRecord(g_pt_ev[2 * s], g_stream);
  return s;
}

void gb__pass_end(int slot) {
  if (slot >= 0) cudaEventRecord(g_pt_ev[2 * slot + 1], g_stream);
}

// Tensor maps (TMA descriptors) for the pipelined strided passes, cached by
// argument set.  The encode entry point is taken from the driver through the
// runtime, so nothing links libcuda directly.
struct TmapKey {
  const void *base;
  long outer, n, inner;
  int fp32, bz, rows;
};
static TmapKey g_tm_key[32];
static CUtensorMap g_tm_val[32];
static int g_tm_used = 0, g_tm_next = 0;
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int gb__tmap_lines(CUtensorMap *out, const void *base, long outer, long n, long inner, int fp32, int bz, int rows) {
  for (int i = 0; i < g_tm_used; i++) {
    const TmapKey &k = g_tm_key[i];
    if (k.base == base && k.outer == outer && k.n == n && k.inner == inner && k.fp32 == fp32 && k.bz == bz &&
        k.rows == rows) {
      *out = g_tm_val[i];
      return 0;
    }
  }
  if (!g_encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess)
      return gb__set_error(1030, "tensor map: cuTensorMapEncodeTiled unavailable");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000) fn;
  }
  const cuuint64_t esz = fp32 ? 4 : 8;
  const cuuint64_t dims[3] = {(cuuint64_t) (2 * inner), (cuuint64_t) n, (cuuint64_t) outer};
  const cuuint64_t strides[2] = {(cuuint64_t) (2 * inner) * esz, (cuuint64_t) (2 * inner) * esz * (cuuint64_t) n};
  const cuuint32_t box[3] = {(cuuint32_t) (2 * bz), (cuuint32_t) rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap m;
  const CUresult r = g_encode(&m, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                              (void *) base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return gb__set_error(1031, "tensor map: encode failed");
  const int slot = g_tm_used < 32 ? g_tm_used++ : (g_tm_next++ & 31);
  g_tm_key[slot] = TmapKey{base, outer, n, inner, fp32, bz, rows};
  g_tm_val[slot] = m;
  *out = m;
  return 0;
}

// ------------------------------------------------------------ device status
//
// One small device block holds the status words of the bounded device-side
// waits (GB_STATUS_PASS: the pipelined pass's copy wait and the plane chain's
// dependency wait; GB_STATUS_CN: the line solver's copy wait;
// GB_STATUS_BATCH: the batch kernel's grid barrier) next to the reduction
// result slot, so a reduction brings its result and the status back in one
// device-to-host copy.  Every host sync point of this layer (gb_synchronize,
// gb_d2h, reductions) reads the status and latches a nonzero word into
// gb_last_error() (code GB_ERR_DEVICE_WAIT), so a wait that gave up is
// reported at the next read of any result instead of leaving wrong values
// unnoticed.  gb_clear_error() clears the words again.

static IoBlock *io_block(void) {
  if (!g_io) {
    if (cudaMalloc(&g_io, sizeof(IoBlock)) != cudaSuccess) {
      cudaGetLastError();
      g_io = nullptr;
      gb__set_error(2, "device status block");
      return nullptr;
    }
    if (cudaHostAlloc(&g_io_host, sizeof(IoBlock), cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      g_io_host = (IoBlock *) calloc(1, sizeof(IoBlock));
    }
    cudaMemsetAsync(g_io, 0, sizeof(IoBlock), g_stream);
  }
  return g_io;
}

int *gb__status(int word) {
  IoBlock *io = io_block();
  return (io && word >= 0 && word < GB_STATUS_WORDS) ? &io->status[word] : nullptr;
}

void *gb__result_slot(void) {
  IoBlock *io = io_block();
  return io ? (void *) io->result : nullptr;
}

static int status_error(const int *st) {
  if (!(st[GB_STATUS_PASS] | st[GB_STATUS_CN] | st[GB_STATUS_BATCH])) return 0;
  char msg[160];
  snprintf(msg, sizeof(msg), "a device-side wait gave up (line passes %d, CN sweeps %d, batch barrier %d)",
           st[GB_STATUS_PASS], st[GB_STATUS_CN], st[GB_STATUS_BATCH]);
  return gb__set_error(GB_ERR_DEVICE_WAIT, msg);
}

int gb__read_result(void *host, size_t bytes) {
  if (!io_block()) return g_err;
  cudaError_t e = cudaMemcpyAsync(g_io_host, g_io, sizeof(IoBlock), cudaMemcpyDeviceToHost, g_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "result copy");
  memcpy(host, g_io_host->result, bytes < sizeof(g_io_host->result) ? bytes : sizeof(g_io_host->result));
  return status_error(g_io_host->status);
}

// Status words only (after the stream has drained); no-op before the block
// exists, since nothing can have written it.
static int check_status(void) {
  if (!g_io) return 0;
  cudaError_t e = cudaMemcpyAsync(g_io_host->status, g_io->status, sizeof(int) * GB_STATUS_WORDS,
                                  cudaMemcpyDeviceToHost, g_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) return gb__set_error((int) e, "status copy");
  return status_error(g_io_host->status);
}

static int status_word(int word, int reset) {
  if (!g_io) return 0;
  int h = 0;
  cudaStreamSynchronize(g_stream);
  cudaMemcpy(&h, &g_io->status[word], sizeof(int), cudaMemcpyDeviceToHost);
  if (reset) cudaMemset(&g_io->status[word], 0, sizeof(int));
  return h;
}

int *gb__pass_errflag(void) { return gb__status(GB_STATUS_PASS); }

extern "C" int gb_pass_error_flag(int reset) { return status_word(GB_STATUS_PASS, reset); }
int gb__status_word(int word, int reset) { return status_word(word, reset); }

extern "C" unsigned gb_wait_limit(unsigned polls) {
  const unsigned old = g_wait_limit;
  g_wait_limit = polls;
  return old;
}
unsigned gb__wait_limit(unsigned dflt) { return g_wait_limit ? g_wait_limit : dflt; }

static int g_chain_lag_pct = 200;
int gb__chain_lag_pct(void) { return g_chain_lag_pct; }
extern "C" int gb_chain_lag(int pct) {
  const int old = g_chain_lag_pct;
  if (pct >= 0) g_chain_lag_pct = pct;
  return old;
}

static int g_pipe_on = 1;
namespace gbfft {
int pipe_enabled() { return g_pipe_on; }
}  // namespace gbfft
extern "C" int gb_pass_pipeline(int on) {
  const int old = g_pipe_on;
  if (on >= 0) g_pipe_on = on ? 1 : 0;
  return old;
}

static int g_plane_on = 1;
namespace gbfft {
int plane_enabled() { return g_plane_on; }
}  // namespace gbfft
extern "C" int gb_plane_passes(int on) {
  const int old = g_plane_on;
  if (on >= 0) g_plane_on = on > 3 ? 3 : on;
  return old;
}

extern "C" int gb_pass_timing_report(double *ms, long *count, int nkinds) {
  for (int k = 0; k < nkinds; k++) {
    ms[k] = 0.0;
    count[k] = 0;
  }
  cudaStreamSynchronize(g_stream);
  for (int s = 0; s < g_pt_used; s++) {
    float e = 0.f;
    if (cudaEventElapsedTime(&e, g_pt_ev[2 * s], g_pt_ev[2 * s + 1]) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    const int k = g_pt_kind[s];
    if (k >= 0 && k < nkinds) {
      ms[k] += e;
      count[k]++;
    }
  }
  return g_pt_used;
}

// ------------------------------------------------------------ conversions

template <typename A, typename B> __global__ void k_convert(B *__restrict__ dst, const A *__restrict__ src, size_t n) {
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = (B) src[i];
}

static unsigned grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b > 148u * 32u) b = 148u * 32u;
  if (b < 1) b = 1;
  return (unsigned) b;
}

extern "C" int gb_convert_f64_to_f32(void *dst, const void *src, size_t n) {
  k_convert<double, float><<<grid_for(n, 256), 256, 0, g_stream>>>((float *) dst, (const double *) src, n);
  GB_CHECK_LAUNCH("convert f64->f32");
  return 0;
}

extern "C" int gb_convert_f32_to_f64(void *dst, const void *src, size_t n) {
  k_convert<float, double><<<grid_for(n, 256), 256, 0, g_stream>>>((double *) dst, (const float *) src, n);
  GB_CHECK_LAUNCH("convert f32->f64");
  return 0;
}

extern "C" int gb_upload_f64_as_f32(void *dev32, const void *host64, size_t n) {
  void *st = gb__scratch(GB_SCR_STAGE, n * sizeof(double));
  if (!st) return gb_last_error();
  if (gb_h2d(st, host64, n * sizeof(double))) return g_err;
  return gb_convert_f64_to_f32(dev32, st, n);
}

extern "C" int gb_download_f32_as_f64(void *host64, const void *dev32, size_t n) {
  void *st = gb__scratch(GB_SCR_STAGE, n * sizeof(double));
  if (!st) return gb_last_error();
  if (gb_convert_f32_to_f64(st, dev32, n)) return g_err;
  return gb_d2h(host64, st, n * sizeof(double));
}

// ---------------------------------------------------------------- twiddles

// exp(-2 pi i m / n) for m < n, rounded from extended precision on the host.
const void *gb__twiddles(long n, int prec) {
  int lg = 0;
  while ((1L << lg) < n) lg++;
  if ((1L << lg) != n || lg < 1 || lg > 12) {
    gb__set_error(1002, "twiddles: unsupported length");
    return nullptr;
  }
  Twiddle &t = g_tw[lg];
  if (!t.d64) {
    double2 *h64 = (double2 *) malloc(sizeof(double2) * (size_t) n);
    float2 *h32 = (float2 *) malloc(sizeof(float2) * (size_t) n);
    for (long m = 0; m < n; m++) {
      long double a = 6.283185307179586476925286766559005768L * (long double) m / (long double) n;
      double c = (double) cosl(a), s = -(double) sinl(a);
      h64[m] = make_double2(c, s);
      h32[m] = make_float2((float) c, (float) s);
    }
    if (cudaMalloc(&t.d64, sizeof(double2) * (size_t) n) != cudaSuccess ||
        cudaMalloc(&t.d32, sizeof(float2) * (size_t) n) != cudaSuccess) {
      cudaGetLastError();
      free(h64);
      free(h32);
      gb__set_error(2, "twiddles cudaMalloc");
      return nullptr;
    }
    cudaMemcpy(t.d64, h64, sizeof(double2) * (size_t) n, cudaMemcpyHostToDevice);
    cudaMemcpy(t.d32, h32, sizeof(float2) * (size_t) n, cudaMemcpyHostToDevice);
    free(h64);
    free(h32);
  }
  return prec == GB_FP32 ? t.d32 : t.d64;
}
