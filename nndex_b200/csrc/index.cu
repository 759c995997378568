// index.cu — the CUDA backend object (CudaIndex) and the C ABI declared in include/nndex_cuda.h.
//
// Mirrors nndex's backend contract: GpuIndex::new / search / search_batch / adapter info
// (src/gpu.rs:138-309, 321-430, 974-1010) behind NNdex::new / search / search_batch
// (src/lib.rs:185-402), with the reference's validation order and error variants
// (src/lib.rs:107-145, 433-450). The device holds the whole normalised base; queries are
// normalised on the device (K1) and scored by the fused scan (K2) + merge.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "index.h"
#include "internal.h"

namespace nndex {

static std::atomic<uint64_t> g_launches{0};
static std::atomic<uint64_t> g_alloc_epoch{0};
static std::atomic<uint32_t> g_fail_allocs{0};  // host-side fault injection: allocations to fail
bool take_injected_alloc_failure() {
    uint32_t n = g_fail_allocs.load(std::memory_order_relaxed);
    while (n > 0 && !g_fail_allocs.compare_exchange_weak(n, n - 1, std::memory_order_relaxed)) {
    }
    return n > 0;
}
void inject_alloc_failures(uint32_t n) { g_fail_allocs.store(n, std::memory_order_relaxed); }
static thread_local cudaStream_t t_scratch_stream = nullptr;
void set_scratch_stream(cudaStream_t s) { t_scratch_stream = s; }
cudaStream_t scratch_stream() { return t_scratch_stream; }
cudaError_t regrow_raw(void** p, size_t bytes) {
    if (bytes == 0) bytes = 1;
    cudaStream_t s = t_scratch_stream;
    if (!s) {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc(p, bytes);
    }
    // never inside a stream capture: the allocation would become a node of a graph that may be
    // discarded (the caller then runs the batch without a graph)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return cudaErrorStreamCaptureUnsupported;
    if (*p) cudaFreeAsync(*p, s);
    *p = nullptr;
    return cudaMallocAsync(p, bytes, s);
}
uint64_t alloc_epoch() { return g_alloc_epoch.load(std::memory_order_acquire); }
void bump_alloc_epoch() { g_alloc_epoch.fetch_add(1, std::memory_order_acq_rel); }
bool sync_check_enabled() {
    static const bool on = [] {
        const char* v = getenv("NNDEX_SYNC_CHECK");
        return v && v[0] == '1';
    }();
    return on;
}
static thread_local char t_launch_note[256];
void set_launch_note(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(t_launch_note, sizeof(t_launch_note), fmt, ap);
    va_end(ap);
}
void count_launch_at(const char* file, int line, uint32_t n) {
    g_launches.fetch_add(n, std::memory_order_relaxed);
    if (!sync_check_enabled()) return;
    static std::atomic<bool> reported{false};
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess && !reported.exchange(true))
        std::fprintf(stderr, "nndex: %s (%d) after the launch at %s:%d [%s]\n", cudaGetErrorString(e),
                     static_cast<int>(e), file, line, t_launch_note);
    t_launch_note[0] = 0;
}
uint64_t kernel_launches_total() { return g_launches.load(std::memory_order_relaxed); }

static thread_local std::string t_error;

int set_error(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_error = buf;
    return code;
}
void clear_error() { t_error.clear(); }
const char* last_error() { return t_error.c_str(); }

int cuda_error(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: %s: out of device memory", what);
    return set_error(NNDEX_ERR_CUDA, "cuda execution error: %s: %s", what, cudaGetErrorString(e));
}

// NNdexError Display strings (src/lib.rs:109-138).
int err_shape(uint64_t rows, uint64_t dims, uint64_t values) {
    return set_error(NNDEX_ERR_SHAPE_MISMATCH, "matrix shape mismatch: rows=%llu, dims=%llu, values=%llu",
                     (unsigned long long)rows, (unsigned long long)dims, (unsigned long long)values);
}
int err_query_dims(uint64_t expected, uint64_t found) {
    return set_error(NNDEX_ERR_QUERY_DIMS, "query dimensionality mismatch: expected %llu, found %llu",
                     (unsigned long long)expected, (unsigned long long)found);
}
int err_topk() { return set_error(NNDEX_ERR_INVALID_TOPK, "top-k must be greater than zero"); }
int err_code(int code) {
    switch (code) {
        case NNDEX_ERR_NON_FINITE: return set_error(code, "all input values must be finite");
        case NNDEX_ERR_ZERO_NORM: return set_error(code, "encountered a zero-norm vector");
        default: return set_error(code, "cuda execution error: device status %d", code);
    }
}

// src/lib.rs:433-442 validate_matrix_shape (saturating multiply).
bool shape_ok(uint64_t n_values, uint64_t rows, uint64_t dims) {
    if (rows == 0 || dims == 0) return false;
    unsigned __int128 p = static_cast<unsigned __int128>(rows) * dims;
    const uint64_t sat = p > UINT64_MAX ? UINT64_MAX : static_cast<uint64_t>(p);
    return sat == n_values;
}

static thread_local int t_encode_result = 0;  // the last encode's CUresult on this thread

static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, uint32_t elem_bytes, const void* base,
                    uint64_t inner, uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                    uint32_t box_outer, CUtensorMapSwizzle swizzle) {
    auto fn = get_encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t es[2] = {1, 1};
    (void)elem_bytes;
    CUresult r = fn(map, dtype, 2, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    t_encode_result = static_cast<int>(r);
    return r == CUDA_SUCCESS;
}
int last_encode_result() { return t_encode_result; }

// ---- device buffers ------------------------------------------------------------------------

template <class T>
static int grow_device(T*& p, size_t& cap, size_t n, const char* what) {
    if (n <= cap && p) return NNDEX_OK;
    bump_alloc_epoch();
    cap = 0;
    void* raw = p;
    cudaError_t e = take_injected_alloc_failure() ? cudaErrorMemoryAllocation
                                                  : regrow_raw(&raw, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaErrorMemoryAllocation && raw) cudaFree(raw);  // an injected failure frees it too
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_error(e, what);
    }
    p = static_cast<T*>(raw);
    cap = n;
    return NNDEX_OK;
}
// Pinned buffers grow geometrically from 4,096 elements: releasing one (cudaFreeHost) waits for
// the device, which in a serving slot means waiting for the other slots' batches too, so they are
// replaced as rarely as possible.
template <class T>
static int grow_host(T*& p, size_t& cap, size_t n, const char* what) {
    if (n <= cap && p) return NNDEX_OK;
    bump_alloc_epoch();
    if (p) cudaFreeHost(p);
    p = nullptr;
    const size_t want = std::max<size_t>({n, cap * 2, 4096});
    cap = 0;
    cudaError_t e = take_injected_alloc_failure()
                        ? cudaErrorMemoryAllocation
                        : cudaMallocHost(reinterpret_cast<void**>(&p), want * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_error(e, what);
    }
    cap = want;
    return NNDEX_OK;
}

void CudaIndex::scan_event_begin(cudaStream_t s, cudaEvent_t& a) {
    a = nullptr;
    if (!scan_timing) return;
    if (scan_events_used == scan_events.size()) {
        cudaEvent_t x, y;
        if (cudaEventCreate(&x) != cudaSuccess) return;
        if (cudaEventCreate(&y) != cudaSuccess) {
            cudaEventDestroy(x);
            return;
        }
        scan_events.emplace_back(x, y);
    }
    a = scan_events[scan_events_used].first;
    cudaEventRecord(a, s);
}

void CudaIndex::scan_event_end(cudaStream_t s, cudaEvent_t a) {
    if (!a) return;
    cudaEventRecord(scan_events[scan_events_used].second, s);
    ++scan_events_used;
}

void CudaIndex::drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
}

CudaIndex::~CudaIndex() {
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    drop_graphs();
    for (auto& p : scan_events) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    if (owns_base) cudaFree(d_base);
    cudaFree(d_qraw);
    cudaFree(d_qn);
    cudaFree(d_ws);
    cudaFree(d_res);
    cudaFree(d_err);  // d_status lives in the same allocation
    cudaFree(d_part_keys);
    cudaFree(d_part_done);
    cudaFreeHost(h_q);
    cudaFreeHost(h_res);
    cudaFreeHost(h_flags);
    if (owns_base) cudaFree(d_base_bf16);
    if (owns_base) cudaFree(d_base_fp8);
    if (owns_base) cudaFree(d_res16);
    if (owns_base) cudaFree(d_res8);
    if (owns_base) cudaFree(d_row_scale);
    if (owns_base) cudaFree(d_tile_scale);
    cudaFree(d_q_bf16);
    cudaFree(d_q_fp8);
    cudaFree(d_q_scale);
    cudaFree(d_q_resid);
    if (owns_base) cudaFree(d_tfnorm);
    cudaFree(d_serr);
    cudaFree(d_serr_acc);
    cudaFreeHost(h_serr_acc);
    cudaFree(d_fbq);
    cudaFree(d_fbn);
    cudaFreeHost(h_fbn);
    cudaFree(d_thr);
    cudaFree(d_cand_idx);
    cudaFree(d_cand_sim);
    cudaFree(d_cand_cnt);
    cudaFree(d_cert);
    cudaFree(d_qsub);
    cudaFree(d_fb_idx);
    cudaFree(d_fb_sim);
    cudaFree(d_fb_cnt);
    cudaFree(d_kth);
    cudaFree(d_floor);
    cudaFree(d_rslots);
    cudaFree(d_ids);
    cudaFree(d_q2_lp);
    cudaFree(d_q2_resid);
    cudaFree(d_q2_scale);
    cudaFree(d_q2_thr);
    cudaFree(d_rows2);
    cudaFree(d_cnt2);
    cudaFree(d_ok2);
    cudaFreeHost(h_ids);
    cudaFreeHost(h_ok2);
    cudaFreeHost(h_cert);
    if (done_ev) cudaEventDestroy(done_ev);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

int CudaIndex::ensure_query_capacity(uint64_t nq) {
    int st;
    if ((st = grow_device(d_qraw, cap_qraw, nq * dims, "query buffer"))) return st;
    if ((st = grow_device(d_qn, cap_qn, nq * ds, "query buffer"))) return st;
    if ((st = grow_host(h_q, cap_hq, nq * dims, "pinned query buffer"))) return st;
    return NNDEX_OK;
}

int CudaIndex::ensure_result_capacity(uint64_t nq, uint64_t kcap) {
    int st;
    const size_t bi = nq * kcap * sizeof(uint64_t), bs = nq * kcap * sizeof(float), bc = nq * sizeof(uint32_t);
    res_bytes = bi + bs + bc;
    if ((st = grow_device(d_res, cap_res, res_bytes, "result buffer"))) return st;
    if ((st = grow_host(h_res, cap_hres, res_bytes, "pinned result buffer"))) return st;
    d_idx = reinterpret_cast<uint64_t*>(d_res);
    d_sim = reinterpret_cast<float*>(d_res + bi);
    d_cnt = reinterpret_cast<uint32_t*>(d_res + bi + bs);
    h_idx = reinterpret_cast<uint64_t*>(h_res);
    h_sim = reinterpret_cast<float*>(h_res + bi);
    h_cnt = reinterpret_cast<uint32_t*>(h_res + bi + bs);
    return NNDEX_OK;
}

// Workspace of the split merge (merge_parts(per_query, k, nq) blocks per query), into m.
int CudaIndex::merge_workspace(uint64_t per_query, uint32_t nq, uint32_t k, MergeArgs& m, cudaStream_t s) {
    const uint32_t parts = merge_parts(per_query, k, nq);
    if (parts <= 1) return NNDEX_OK;
    int st;
    if ((st = grow_device(d_part_keys, cap_part_keys, static_cast<size_t>(nq) * parts * k, "merge workspace")))
        return st;
    // counters start at zero: clear them whenever the buffer is (re)allocated (a new allocation
    // may return the old address, so compare capacities, not pointers)
    const size_t cap_before = cap_part_done;
    if ((st = grow_device(d_part_done, cap_part_done, nq, "merge workspace"))) return st;
    if (cap_part_done != cap_before) cudaMemsetAsync(d_part_done, 0, cap_part_done * sizeof(uint32_t), s);
    m.part_keys = d_part_keys;
    m.part_done = d_part_done;
    return NNDEX_OK;
}

// Enqueue the exact FP32 top-k of `nq` normalised queries (d_queries, stride ds) into the
// device outputs. Workspace is the index's own (grown on demand).
int CudaIndex::enqueue_exact_fp32(const float* d_queries, uint32_t nq, uint32_t k, uint32_t out_stride,
                                  uint64_t* o_idx, float* o_sim, uint32_t* o_cnt, cudaStream_t s) {
    ScanPlan plan;
    if (!plan_scan_fp32(nq, static_cast<uint32_t>(ds), k, rows, sm_count, smem_optin, plan))
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: k=%u above the fused top-k limit %u", k,
                         kMaxFusedK);
    const uint64_t per_query = static_cast<uint64_t>(plan.ctas_per_group) * k;
    int st = grow_device(d_ws, cap_ws, per_query * nq, "scan workspace");
    if (st) return st;
    ScanArgs a;
    a.tmap = &tmap_f32;
    a.tmap_tile = &tmap_f32_176;
    a.tmap_112 = &tmap_f32_112;
    a.queries = d_queries;
    a.nq = nq;
    a.dq = static_cast<uint32_t>(ds);
    a.rows = rows;
    a.k = k;
    a.ws_keys = d_ws;
    a.status = d_status;
    cudaEvent_t ev_a = nullptr;
    scan_event_begin(s, ev_a);
    cudaError_t e = launch_scan_fp32(a, plan, s);
    scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "scan launch");
    MergeArgs m;
    m.ws_keys = d_ws;
    m.nq = nq;
    m.per_query = per_query;
    m.k = k;
    m.out_stride = out_stride;
    m.idx_out = o_idx;
    m.sim_out = o_sim;
    m.count_out = o_cnt;
    if ((st = merge_workspace(per_query, nq, k, m, s))) return st;
    e = launch_merge_topk(m, s);
    if (e != cudaSuccess) return cuda_error(e, "merge launch");
    stats.kernel_launches += 2;
    stats.path = 1;
    stats.rows_scanned += rows * nq;
    stats.scan_qb = plan.qb;
    stats.scan_wide = plan.wide;
    return NNDEX_OK;
}

// Prepare `nq` raw queries already in d_qraw (mode per K1) into d_qn.
int CudaIndex::enqueue_query_prep(uint64_t nq, int mode, cudaStream_t s) {
    PrepArgs p;
    p.src = d_qraw;
    p.rows = nq;
    p.dims = static_cast<uint32_t>(dims);
    p.out = d_qn;
    p.out_stride = static_cast<uint32_t>(ds);
    p.mode = mode;
    p.err = d_err;
    p.sm_count = sm_count;
    launch_prep_rows(p, s);
    stats.kernel_launches += 1;
    return NNDEX_OK;
}

int CudaIndex::check_device_words() {
    // h_flags[0] = err word, h_flags[1] = status word (copied with the results).
    const uint64_t err = h_flags[0];
    const uint32_t status = static_cast<uint32_t>(h_flags[1]);
    if (err != ~0ull) return err_code(static_cast<int>(err & 0xFF));
    if (status == kStatusTimeout)
        return set_error(NNDEX_ERR_TIMEOUT, "cuda execution error: a bounded device wait timed out");
    if (status != 0) return set_error(NNDEX_ERR_CUDA, "cuda execution error: device status %u", status);
    return NNDEX_OK;
}

// ---- path choice (rules by batch size, k and the index's copies) ----------------------------

int CudaIndex::choose_path(uint64_t nq, uint64_t kcap) const {
    const bool has16 = d_base_bf16 != nullptr, has8 = d_base_fp8 != nullptr;
    auto tc_ok = [&](bool fp8) {
        const TcPlan p1 = plan_tc(kcap, fp8);
        return p1.kp >= kcap && p1.kp > 0 && plan_tc(0, fp8).stages > 0;
    };
    // Small batches (plan_tf32's range): the TF32 candidate scan, which reads the same FP32 base and
    // returns the same bits as the FP32 scan at the HBM rate, where the FP32 scan is bound by its
    // FMA issue.
    const int fp32_path = plan_tf32(nq, kcap).kp ? 6 : 1;
    switch (precision) {
        case NNDEX_PRECISION_FP32: return fp32_path;
        case NNDEX_PRECISION_BF16: return (has16 && tc_ok(false)) ? 2 : 1;
        case NNDEX_PRECISION_FP8: return (has8 && tc_ok(true)) ? 3 : 1;
        default:
            // FP32 streaming is HBM-bound at small batches; the tensor cores win from a few dozen
            // queries per batch (the scan becomes compute-bound in FP32).
            if (nq >= 64) {
                if (has16 && tc_ok(false)) return 2;
                if (has8 && tc_ok(true)) return 3;
            }
            return fp32_path;
    }
}

CudaIndex::Tf32Plan CudaIndex::plan_tf32(uint64_t nq, uint64_t kcap) const {
    Tf32Plan p;
    static const uint32_t min_q = [] {
        const char* v = getenv("NNDEX_TF32_MIN_QUERIES");  // measurement override of the batch rule
        return v ? static_cast<uint32_t>(atoi(v)) : 9u;
    }();
    static const bool off = [] {
        const char* v = getenv("NNDEX_TF32_SCAN");  // 0: small batches always take the FP32 scan
        return v && v[0] == '0';
    }();
    if (off || !d_tfnorm || nq < std::max<uint32_t>(min_q, 1) || nq > 16 || kcap == 0 || kcap > 448) return p;
    // k′: 2.5 k rounded up to 32, at least k + 64 and at most 512, so that the exact k-th score
    // clears the k′-th bound on clustered data (on a 1,024-centre mixture of 1M × 768 rows the
    // 100th and 256th scores of a query are ≈ 2.4e-3 apart, twice the bound's typical ε)
    const uint64_t kp = std::min<uint64_t>(512, (std::max<uint64_t>(kcap * 5 / 2, kcap + 64) + 31) / 32 * 32);
    if (rows < 4 * kp || rows > 0xFFFFFFFFull) return p;
    // Each CTA lists a quarter of k′ (at least 32): the k′ best of a query come from all 148 CTAs,
    // and the rows a full list left out score below the largest full-list minimum (the floor),
    // which the certificate then also has to clear.
    const uint32_t kp_cta = static_cast<uint32_t>(std::max<uint64_t>(32, (kp / 4 + 31) / 32 * 32));
    // Room for three tiles of survivors above the list: a selection runs once ≥ 256 keys have
    // accumulated since the last one, not after every tile.
    const uint32_t cap = kp_cta + 3 * 128;
    const uint32_t stages = tf32_stages_for(cap, smem_optin);
    if (!stages) return p;
    p.kp = static_cast<uint32_t>(kp);
    p.kp_cta = kp_cta;
    p.cap = cap;
    p.stages = stages;
    return p;
}

// C of K12's bound, per unit ‖q‖‖x‖:
//   the tensor core's FP32 accumulation of ds exact TF32 products (each added with up to one FP32
//   rounding, 4× margin, as for the BF16 scan):                              4·ds·2⁻²³
//   the FP32 scan's own rounding (eight chains of ds/8 FMAs, then 3 adds):  (ds/8 + 3)·2⁻²⁴
//   the rounding of u = s̃ + ε:                                             2⁻²²
float CudaIndex::tf32_c_norm() const {
    const double d = static_cast<double>(ds);
    return static_cast<float>((4.0 * d * std::ldexp(1.0, -23) + (d / 8.0 + 3.0) * std::ldexp(1.0, -24) +
                               std::ldexp(1.0, -22)) * 1.01);
}

// For unit rows and queries ‖d_v‖ < 2⁻¹⁰: ε < 2·2⁻¹⁰ + 2⁻²⁰ + C.
float CudaIndex::tf32_eps() const {
    return static_cast<float>((2.0 * std::ldexp(1.0, -10) + std::ldexp(1.0, -20) + tf32_c_norm()) * 1.01);
}

// IVF batches: the tensor-core list scan (5) from a few dozen queries, when the index's precision
// allows low-precision scoring and k fits its pass-1 heaps; else the FP32 list scan (4).
int CudaIndex::ivf_path(uint64_t nq, uint64_t kcap) const {
    if (precision == NNDEX_PRECISION_FP32 || nq < 64 || !ivf || !ivf->d_reordered16) return 4;
    // The tensor-core list scan scores 128-query blocks per list chunk (≤ 4096 rows). With few
    // queries per probed list and short lists its items are small and their fixed cost dominates:
    // on 2M × 384 (nlist 1414, lists of ≈ 1,400 rows) with 1024 queries, nprobe 8 (≈ 6 queries per
    // list) runs faster on the FP32 list scan (489k vs 350k q/s), nprobe 32 (≈ 23) and 64 (≈ 46)
    // on the tensor cores (345k vs 269k, 324k vs 174k). With long lists (5M × 512, nlist 512, lists
    // of ≈ 9,800 rows) the tensor cores win from 64 queries on (serving at saturation: 157k vs 132k
    // q/s). So: the FP32 list scan when a probed list serves fewer than 12 queries on average and
    // the average list is shorter than one 4096-row chunk.
    const uint64_t np0 = ivf_scratch.nprobe ? ivf_scratch.nprobe : ivf_choose_nprobe(ivf->nlist, kcap, rows);
    const double per_list = static_cast<double>(nq) * static_cast<double>(std::min<uint64_t>(np0, ivf->nlist)) /
                            static_cast<double>(ivf->nlist);
    static const double min_per_list = [] {
        const char* v = getenv("NNDEX_IVF_TC_MIN_PER_LIST");  // measurement override of the rule
        return v ? atof(v) : 12.0;
    }();
    if (per_list < min_per_list && rows / ivf->nlist < 4096) return 4;
    const TcPlan p1 = plan_tc(kcap, false);
    return (p1.kp >= kcap && p1.kp > 0 && plan_tc(0, false).stages > 0) ? 5 : 4;
}

uint32_t CudaIndex::tc_chunks(bool fp8) const {
    return static_cast<uint32_t>((fp8 ? kf8 : kb16 * 2) / 128);
}

// Shared-memory plan of a tensor-core pass. kcap = 0 plans pass 2 (no heaps). Pass 1 wants
// k′ = max(32, 2k) heap entries per query (enough that most queries certify) beside a 4-deep ring
// with the query block resident; it gives up, in order: the ring depth for a k′ that still holds k
// (queries that do not certify take the threshold pass), then the resident query block (its slabs
// then travel with every ring stage), then the k′ margin (k′ = k).
CudaIndex::TcPlan CudaIndex::plan_tc(uint64_t kcap, bool fp8) const {
    const uint32_t nchunks = tc_chunks(fp8);
    TcPlan out;
    if (kcap == 0) {
        out.stages = tc_stages_for(nchunks, 0, fp8, false, smem_optin);
        if (!out.stages) {
            out.stream_a = true;
            out.stages = tc_stages_for(nchunks, 0, fp8, true, smem_optin);
        }
        return out;
    }
    auto largest = [&](bool stream_a, bool four) {
        uint32_t best = 0;
        for (uint32_t kp = 8; kp <= 2048; kp += 8) {
            const uint32_t stg = tc_stages_for(nchunks, kp, fp8, stream_a, smem_optin);
            if (four ? stg == 4 : stg != 0) best = kp;
        }
        return best;
    };
    const uint32_t kmax4 = largest(false, true), kmax = largest(false, false), kmax_s = largest(true, false);
    uint32_t want = rerank_width ? rerank_width : static_cast<uint32_t>(std::max<uint64_t>(32, 2 * kcap));
    if (want > rows) want = static_cast<uint32_t>(rows);
    uint32_t kp = want;
    if (kp > kmax4 && kcap <= kmax4 && !rerank_width) kp = kmax4;
    if (kp > kmax) kp = kmax;
    if (kp >= kcap && kp > 0) {
        out.kp = kp;
        out.stages = tc_stages_for(nchunks, kp, fp8, false, smem_optin);
        return out;
    }
    kp = std::min(want, kmax_s);  // streamed query slabs
    if (kp < kcap) return out;    // no tensor-core plan: the FP32 scan serves this k
    out.kp = kp;
    out.stream_a = true;
    out.stages = tc_stages_for(nchunks, kp, fp8, true, smem_optin);
    return out;
}

int CudaIndex::enqueue_prep_queries(const float* d_raw, uint64_t n, int mode, int path, cudaStream_t s) {
    int st;
    PrepArgs p;
    p.src = d_raw;
    p.rows = n;
    p.dims = static_cast<uint32_t>(dims);
    p.out = d_qn;
    p.out_stride = static_cast<uint32_t>(ds);
    p.mode = mode;
    p.err = d_err;
    p.sm_count = sm_count;
    if (path == 2 || path == 3 || path == 5) {
        const uint64_t nq_alloc = (n + 127) / 128 * 128;
        if ((st = grow_device(d_q_resid, cap_q_resid, n, "query buffer"))) return st;
        if (path == 2 || path == 5) {
            const bool grew = nq_alloc * kb16 > cap_q_bf16;
            if ((st = grow_device(d_q_bf16, cap_q_bf16, nq_alloc * kb16, "query buffer"))) return st;
            if (grew) cudaMemsetAsync(d_q_bf16, 0, cap_q_bf16 * sizeof(__nv_bfloat16), s);
            p.out_bf16 = d_q_bf16;
            p.bf16_stride = static_cast<uint32_t>(kb16);
            p.resid_bf16 = d_q_resid;
        } else {
            const bool grew = nq_alloc * kf8 > cap_q_fp8;
            if ((st = grow_device(d_q_fp8, cap_q_fp8, nq_alloc * kf8, "query buffer"))) return st;
            if (grew) cudaMemsetAsync(d_q_fp8, 0, cap_q_fp8, s);
            if ((st = grow_device(d_q_scale, cap_q_scale, n, "query buffer"))) return st;
            p.out_fp8 = d_q_fp8;
            p.fp8_stride = static_cast<uint32_t>(kf8);
            p.fp8_scale = d_q_scale;
            p.resid_fp8 = d_q_resid;
        }
    }
    launch_prep_rows(p, s);
    stats.kernel_launches += 1;
    return NNDEX_OK;
}

int CudaIndex::enqueue_tc(bool fp8, uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                          cudaStream_t s) {
    int st;
    const TcPlan plan = plan_tc(kcap, fp8);
    const uint32_t kp = plan.kp, stages = plan.stages;
    if (!stages || kp < kcap) return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: k'=%u does not fit", kp);
    const uint32_t nqb = (n + 127) / 128;
    uint64_t nranges = 0, range_rows = 0;
    tc_ranges(nqb, nranges, range_rows);
    const uint64_t per_query = nranges * kp;
    // Autotuned: when the last batch rarely certified in pass 1, pass 1 only has to produce each
    // query's threshold T, and a sample of the rows (every 8th tile) gives a valid one.
    // The tuner's plan may fix it instead (only bases of ≥ 64 tiles are sampled).
    // At k ≥ 64 the rules start sampled: a full pass 1 then carries the largest heaps and almost
    // never certifies (the k′ the shared memory allows is little above k), and the rule's state is
    // shared with the index's small-k batches, which may keep it at 1.
    const uint32_t want = forced_stride ? forced_stride : (kcap >= 64 ? 8u : tc_sample_stride);
    const uint32_t stride = (want > 1 && rows >= 256ull * 64) ? want : 1;
    if ((st = grow_device(d_thr, cap_thr, n, "tc workspace"))) return st;
    if ((st = grow_device(d_ws, cap_ws, per_query * n, "tc workspace"))) return st;
    if ((st = grow_device(d_cand_idx, cap_cand_idx, static_cast<uint64_t>(n) * kp, "tc workspace"))) return st;
    if ((st = grow_device(d_cand_sim, cap_cand_sim, static_cast<uint64_t>(n) * kp, "tc workspace"))) return st;
    if ((st = grow_device(d_cand_cnt, cap_cand_cnt, n, "tc workspace"))) return st;
    if ((st = grow_device(d_cert, cap_cert, n, "tc workspace"))) return st;
    if ((st = grow_device(d_kth, cap_kth, n, "tc workspace"))) return st;
    CUtensorMap tmap_q;
    if ((st = encode_query_tmap(fp8, fp8 ? static_cast<void*>(d_q_fp8) : static_cast<void*>(d_q_bf16), n, &tmap_q)))
        return st;
    cudaMemsetAsync(d_thr, 0, n * sizeof(unsigned long long), s);
    TcArgs a;
    a.tmap_q = &tmap_q;
    a.tmap_b = fp8 ? &tmap_fp8 : &tmap_bf16;
    a.nranges = static_cast<uint32_t>(nranges);
    a.stages = stages;
    a.stream_a = plan.stream_a;
    fill_tc_params(fp8, n, range_rows, a.p);
    a.p.q_resid = d_q_resid;
    a.p.q_scale = fp8 ? d_q_scale : nullptr;
    a.p.kprime = kp;
    a.p.heap_k = stride > 1 ? std::max(1u, std::min(kp, kcap)) : kp;  // a sampled pass 1 only yields T
    a.p.thr_global = d_thr;
    a.p.ws_keys = d_ws;
    a.p.tile_stride = stride;
    last_tc_stride = stride;
    stats.pass1_tile_stride = stride;
    cudaEvent_t ev_a = nullptr;
    scan_event_begin(s, ev_a);
    cudaError_t e = launch_scan_tc(a, fp8, 0, s);
    scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "tensor-core scan launch");
    MergeArgs m;
    m.ws_keys = d_ws;
    m.nq = n;
    m.per_query = per_query;
    m.k = kp;
    m.out_stride = kp;
    m.idx_out = d_cand_idx;
    m.sim_out = d_cand_sim;
    m.count_out = d_cand_cnt;
    if ((st = merge_workspace(per_query, n, kp, m, s))) return st;
    if ((e = launch_merge_topk(m, s)) != cudaSuccess) return cuda_error(e, "merge launch");
    RerankArgs r;
    r.base = d_base;
    r.ds = static_cast<uint32_t>(ds);
    r.queries = d_qn;
    r.cand_idx = d_cand_idx;
    r.cand_sim = d_cand_sim;
    r.cand_cnt = d_cand_cnt;
    r.nq = n;
    r.kp = kp;
    r.k = kcap;
    r.idx_out = o_idx;
    r.sim_out = o_sim;
    r.cnt_out = o_cnt;
    r.cert_out = d_cert;
    r.kth_out = d_kth;
    r.certify = stride == 1;
    if ((e = launch_rerank(r, s)) != cudaSuccess) return cuda_error(e, "rerank launch");
    stats.kernel_launches += 3;
    stats.path = fp8 ? 3 : 2;
    stats.rerank_width = kp;
    stats.rows_scanned += rows * n;
    return NNDEX_OK;
}

// Row ranges of the tensor-core grid: about four waves of CTAs, each range a multiple of the
// 256-row tile. Concurrent CTAs share ranges, so a base tile is read from HBM about once.
void CudaIndex::tc_ranges(uint32_t nqb, uint64_t& nranges, uint64_t& range_rows) const {
    tc_range_split(rows, nqb, static_cast<uint64_t>(sm_count), nranges, range_rows);
}

void CudaIndex::fill_tc_params(bool fp8, uint32_t n, uint64_t range_rows, TcParams& p) const {
    const uint64_t kb = fp8 ? kf8 : kb16;
    p.nq = n;
    p.nchunks = tc_chunks(fp8);
    p.rows = rows;
    p.range_rows = range_rows;
    p.row_scale = fp8 ? d_row_scale : nullptr;
    p.tile_scale = fp8 ? d_tile_scale : nullptr;
    p.row_resid = fp8 ? d_res8 : d_res16;
    p.eps_rows = fp8 ? eps_fp8 : eps_bf16;
    // FP32 accumulation of kb exact products (|Σ| ≤ 1 + ε): kb·2^-23, with a 4× margin.
    p.eps_acc = 4.0f * static_cast<float>(kb) * 1.1920929e-07f;
    p.status = d_status;
}

int CudaIndex::encode_query_tmap(bool fp8, void* buf, uint32_t n, CUtensorMap* map) const {
    const uint64_t nq_alloc = (n + 127) / 128 * 128;
    const bool ok = fp8 ? encode_tmap_2d(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, buf, kf8, nq_alloc, kf8, 128, 128,
                                         CU_TENSOR_MAP_SWIZZLE_128B)
                        : encode_tmap_2d(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, buf, kb16, nq_alloc, kb16 * 2, 64,
                                         128, CU_TENSOR_MAP_SWIZZLE_128B);
    if (!ok)
        return set_error(NNDEX_ERR_CUDA,
                         "cuda execution error: cuTensorMapEncodeTiled failed (queries: %s, %u rows, row length %llu, "
                         "buffer %p, driver result %d)",
                         fp8 ? "FP8" : "BF16", n, (unsigned long long)(fp8 ? kf8 : kb16), buf, last_encode_result());
    return NNDEX_OK;
}

int CudaIndex::ensure_fbn() {
    if (d_fbn) return NNDEX_OK;
    cudaError_t e;
    if ((e = cudaMalloc(&d_fbn, 4 * sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMallocHost(&h_fbn, 4 * sizeof(uint32_t))) != cudaSuccess)
        return cuda_error(e, "fallback buffer");
    return NNDEX_OK;
}

// After pass 1: queries whose certificate held are final. The others run pass 2 (collect every row
// whose upper bound reaches their exact k-th score, rerank exactly) — all on the device, sized for
// the worst case (every query uncertified), the kernels reading the count that the compaction left.
int CudaIndex::enqueue_tc_pass2(bool fp8, uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim,
                                uint32_t* o_cnt, cudaStream_t s) {
    int st;
    const uint32_t cap2 = kSecondPassCap;
    const uint64_t row_bytes = fp8 ? kf8 : kb16 * 2;
    const uint64_t n_alloc = (n + 127) / 128 * 128;
    if ((st = ensure_fbn())) return st;
    if ((st = grow_device(d_ids, cap_ids, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_q2_lp, cap_q2_lp, n_alloc * row_bytes, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_q2_resid, cap_q2_resid, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_q2_scale, cap_q2_scale, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_q2_thr, cap_q2_thr, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_rows2, cap_rows2, static_cast<uint64_t>(n) * cap2, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_cnt2, cap_cnt2, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_ok2, cap_ok2, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_tcfail, cap_tcfail, n, "pass-2 buffer"))) return st;
    if ((st = grow_device(d_rslots, cap_rslots, static_cast<uint64_t>(n) * rerank_chunks(cap2) * kcap,
                          "pass-2 buffer")))
        return st;
    uint32_t* d_m = d_fbn + 1;      // uncertified queries
    uint32_t* d_fail = d_fbn + 2;   // of them, collections that overflowed
    launch_compact_zero_flags(d_cert, n, d_ids, d_m, s);
    cudaError_t e = launch_gather_queries(d_ids, n, fp8 ? static_cast<const void*>(d_q_fp8)
                                                         : static_cast<const void*>(d_q_bf16),
                                          static_cast<uint32_t>(row_bytes), d_q2_lp, d_q_resid, d_q2_resid,
                                          fp8 ? d_q_scale : nullptr, d_q2_scale, d_kth, d_q2_thr, s, d_m);
    if (e != cudaSuccess) return cuda_error(e, "gather launch");
    cudaMemsetAsync(d_cnt2, 0, n * sizeof(uint32_t), s);
    CUtensorMap tmap_q2;
    if ((st = encode_query_tmap(fp8, d_q2_lp, n, &tmap_q2))) return st;
    TcArgs a;
    a.tmap_q = &tmap_q2;
    a.tmap_b = fp8 ? &tmap_fp8 : &tmap_bf16;
    const TcPlan plan2 = plan_tc(0, fp8);
    a.stages = plan2.stages;
    a.stream_a = plan2.stream_a;
    // Two query blocks per CTA (where both fit beside a ring: D ≤ 256 in BF16, 512 in FP8) read half
    // the base bytes per FLOP but run M = 128, N = 128 MMAs, which read as many query bytes from
    // shared memory as base bytes. On 10M × 256 at 4,096 queries that made BF16 7 % slower, and FP8
    // 7 % faster only while the row ranges left SMs idle in a last partial round (the autotuner has
    // taken one block for FP8 since): the rule takes one block, and the autotuner times both.
    // CTA pairs (qb = 3): two CTAs, one query block each, share every 256-row base tile through
    // M = 256 MMAs, so each SM reads half the base bytes per FLOP without narrowing the MMA.
    const uint32_t want_qb = forced_qb ? forced_qb : 1u;
    const uint32_t pair_stages = (want_qb == 2 && n > 128) ? tc_pair_stages_for(tc_chunks(fp8), fp8, smem_optin) : 0;
    const uint32_t cta_pair_stages =
        (want_qb == 3 && n > 128) ? tc_cta_pair_stages_for(tc_chunks(fp8), fp8, smem_optin) : 0;
    if (pair_stages || cta_pair_stages) {
        a.qb = pair_stages ? 2 : 3;
        a.stages = pair_stages ? pair_stages : cta_pair_stages;
        a.stream_a = false;
        a.tmap_b = fp8 ? &tmap_fp8_h : &tmap_bf16_h;
    }
    stats.pass2_query_blocks = a.qb;
    fill_tc_params(fp8, n, 0, a.p);
    a.p.q_resid = d_q2_resid;
    a.p.q_scale = fp8 ? d_q2_scale : nullptr;
    a.p.q_thr = d_q2_thr;
    a.p.cand_rows = d_rows2;
    a.p.cand_cnt = d_cnt2;
    a.p.cap2 = cap2;
    a.p.live_q = d_m;
    a.p.sm_count = static_cast<uint32_t>(sm_count);
    // (query block, row range) items for any count ≤ n: at most 8 per SM plus one per block
    // (tc_range_split: at most 8 rounds, or one range per block)
    a.live_items = 8u * static_cast<uint32_t>(sm_count) + static_cast<uint32_t>(n_alloc / 128) + 1u;
    cudaEvent_t ev_a = nullptr;
    scan_event_begin(s, ev_a);
    e = launch_scan_tc(a, fp8, 1, s);
    scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "tensor-core scan launch (pass 2)");
    e = launch_rerank_collected(d_base, static_cast<uint32_t>(ds), d_qn, d_ids, n, d_rows2, d_cnt2, cap2, kcap,
                                d_q2_thr, d_rslots, o_idx, o_sim, o_cnt, d_ok2, s, false, d_m);
    if (e != cudaSuccess) return cuda_error(e, "rerank launch (pass 2)");
    launch_compact_zero_flags(d_ok2, n, d_tcfail, d_fail, s, d_m);
    stats.kernel_launches += 6;
    last_tc_n = n;
    return NNDEX_OK;
}

int CudaIndex::finish_tc(uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                         cudaStream_t s) {
    const uint32_t m = h_fbn[1], failed_n = h_fbn[2];
    stats.certified = m == 0 ? 1u : 0u;
    stats.second_pass_queries = m;
    // The rule for the next batch (when no tuned plan fixes the stride): a full pass 1 pays off only
    // when it certifies most queries.
    if (!forced_stride) {
        const uint32_t before = tc_sample_stride;
        if (last_tc_stride == 1) tc_sample_stride = (m * 2 > n) ? 8u : 1u;
        else if (m * 2 <= n) tc_sample_stride = 1;
        if (tc_sample_stride != before) drop_graphs();  // a captured batch keeps its stride
    }
    stats.fp32_fallback_queries = failed_n;
    int st;
    if (m) {
        // rows collected by pass 2 (the counts of its m queries, after the batch)
        if ((st = grow_host(h_ok2, cap_hok2, n, "pinned buffer"))) return st;
        cudaMemcpyAsync(h_ok2, d_cnt2, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        const cudaError_t e0 = cudaStreamSynchronize(s);
        if (e0 != cudaSuccess) return cuda_error(e0, "search");
        uint64_t total = 0;
        for (uint32_t i = 0; i < m; ++i) total += std::min<uint32_t>(h_ok2[i], kSecondPassCap);
        stats.pass2_rows += total;
    }
    if (failed_n == 0) return NNDEX_OK;
    // ---- the FP32 scan for queries whose collected set overflowed ----
    if ((st = grow_host(h_ids, cap_hids, n, "pinned buffer"))) return st;
    if ((st = grow_host(h_ok2, cap_hok2, n, "pinned buffer"))) return st;
    cudaMemcpyAsync(h_ids, d_ids, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_ok2, d_tcfail, failed_n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "search");
    std::vector<uint32_t> failed(failed_n);
    for (uint32_t i = 0; i < failed_n; ++i) failed[i] = h_ids[h_ok2[i]];
    return rerun_exact_fp32(failed, kcap, o_idx, o_sim, o_cnt, s);
}

int CudaIndex::rerun_exact_fp32(const std::vector<uint32_t>& qs, uint32_t kcap, uint64_t* o_idx, float* o_sim,
                                uint32_t* o_cnt, cudaStream_t s) {
    int st;
    const uint32_t mf = static_cast<uint32_t>(qs.size());
    if ((st = grow_device(d_qsub, cap_qsub, static_cast<uint64_t>(mf) * ds, "fallback buffer"))) return st;
    for (uint32_t i = 0; i < mf; ++i)
        cudaMemcpyAsync(d_qsub + static_cast<uint64_t>(i) * ds, d_qn + static_cast<uint64_t>(qs[i]) * ds,
                        ds * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if ((st = grow_device(d_fb_idx, cap_fb_idx, static_cast<uint64_t>(mf) * kcap, "fallback buffer"))) return st;
    if ((st = grow_device(d_fb_sim, cap_fb_sim, static_cast<uint64_t>(mf) * kcap, "fallback buffer"))) return st;
    if ((st = grow_device(d_fb_cnt, cap_fb_cnt, mf, "fallback buffer"))) return st;
    const uint32_t path = stats.path;
    if ((st = enqueue_exact_fp32(d_qsub, mf, kcap, kcap, d_fb_idx, d_fb_sim, d_fb_cnt, s))) return st;
    stats.path = path;
    for (uint32_t i = 0; i < mf; ++i) {
        const uint64_t q = qs[i];
        cudaMemcpyAsync(o_idx + q * kcap, d_fb_idx + static_cast<uint64_t>(i) * kcap, kcap * sizeof(uint64_t),
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(o_sim + q * kcap, d_fb_sim + static_cast<uint64_t>(i) * kcap, kcap * sizeof(float),
                        cudaMemcpyDeviceToDevice, s);
        if (o_cnt) cudaMemcpyAsync(o_cnt + q, d_fb_cnt + i, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "search");
    return NNDEX_OK;
}

// K12 (small batches, FP32 precision): the TF32 candidate scan, the merge of each query's per-CTA
// candidates, and the exact rerank with its certificate into the outputs.
int CudaIndex::enqueue_tf32(uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                            cudaStream_t s) {
    int st;
    const Tf32Plan plan = plan_tf32(n, kcap);
    if (!plan.kp) return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: no TF32 scan plan for k=%u", kcap);
    const uint32_t kp = plan.kp;
    const uint32_t ctas = static_cast<uint32_t>(sm_count);
    const uint64_t per_query = static_cast<uint64_t>(ctas) * plan.kp_cta;
    // the FP32 scan that re-runs uncertified queries shares the candidate workspace
    ScanPlan fb_plan;
    if (!plan_scan_fp32(n, static_cast<uint32_t>(ds), kcap, rows, sm_count, smem_optin, fb_plan))
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: no FP32 scan plan for k=%u", kcap);
    const uint64_t fb_per_query = static_cast<uint64_t>(fb_plan.ctas_per_group) * kcap;
    if ((st = grow_device(d_ws, cap_ws, std::max(per_query, fb_per_query) * n, "scan workspace"))) return st;
    if ((st = grow_device(d_qsub, cap_qsub, static_cast<uint64_t>(n) * ds, "fallback buffer"))) return st;
    if ((st = grow_device(d_fbq, cap_fbq, n, "fallback buffer"))) return st;
    if (!d_fbn) {
        cudaError_t e0;
        if ((e0 = cudaMalloc(&d_fbn, 4 * sizeof(uint32_t))) != cudaSuccess ||
            (e0 = cudaMallocHost(&h_fbn, 4 * sizeof(uint32_t))) != cudaSuccess)
            return cuda_error(e0, "fallback buffer");
    }
    if ((st = grow_device(d_cand_idx, cap_cand_idx, static_cast<uint64_t>(n) * kp, "tc workspace"))) return st;
    if ((st = grow_device(d_cand_sim, cap_cand_sim, static_cast<uint64_t>(n) * kp, "tc workspace"))) return st;
    if ((st = grow_device(d_cand_cnt, cap_cand_cnt, n, "tc workspace"))) return st;
    if ((st = grow_device(d_cert, cap_cert, n, "tc workspace"))) return st;
    if ((st = grow_device(d_kth, cap_kth, n, "tc workspace"))) return st;
    if ((st = grow_device(d_floor, cap_floor, n, "tc workspace"))) return st;
    // The queries straight from the prepared buffer: rows past n read as zeros.
    CUtensorMap tmap_q;
    if (!encode_tmap_2d(&tmap_q, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, d_qn, ds, n, ds * sizeof(float), 32, 16,
                        CU_TENSOR_MAP_SWIZZLE_128B))
        return set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed (queries, driver "
                                         "result %d)", last_encode_result());
    Tf32ScanArgs a;
    a.nq = n;
    a.nbox = static_cast<uint32_t>(ds / 32);
    a.ds = static_cast<uint32_t>(ds);
    a.rows = rows;
    a.kp = plan.kp_cta;
    a.cap = plan.cap;
    a.queries = d_qn;
    a.row_norms = d_tfnorm;
    a.c_norm = tf32_c_norm();
    a.evict_first = n <= 16;
    a.ws_keys = d_ws;
    a.floor_keys = d_floor;
    a.status = d_status;
    cudaMemsetAsync(d_floor, 0, n * sizeof(unsigned long long), s);
    cudaEvent_t ev_a = nullptr;
    scan_event_begin(s, ev_a);
    cudaError_t e = launch_scan_tf32(tmap_f32, tmap_q, a, plan.stages, ctas, s);
    scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "TF32 scan launch");
    MergeArgs m;
    m.ws_keys = d_ws;
    m.nq = n;
    m.per_query = per_query;
    m.k = kp;
    m.out_stride = kp;
    m.idx_out = d_cand_idx;
    m.sim_out = d_cand_sim;
    m.count_out = d_cand_cnt;
    if ((st = merge_workspace(per_query, n, kp, m, s))) return st;
    if ((e = launch_merge_topk(m, s)) != cudaSuccess) return cuda_error(e, "merge launch");
    RerankArgs r;
    r.base = d_base;
    r.ds = static_cast<uint32_t>(ds);
    r.queries = d_qn;
    r.cand_idx = d_cand_idx;
    r.cand_sim = d_cand_sim;
    r.cand_cnt = d_cand_cnt;
    r.nq = n;
    r.kp = kp;
    r.k = kcap;
    r.idx_out = o_idx;
    r.sim_out = o_sim;
    r.cnt_out = o_cnt;
    r.cert_out = d_cert;
    r.kth_out = d_kth;
    r.certify = true;
    r.floor_keys = d_floor;  // rows the CTAs' lists left out score below it
    r.fb_ids = d_fbq;
    r.fb_count = d_fbn;
    cudaMemsetAsync(d_fbn, 0, sizeof(uint32_t), s);
    if ((e = launch_rerank(r, s)) != cudaSuccess) return cuda_error(e, "rerank launch");
    // Uncertified queries re-run on the FP32 scan, on the device: the rerank listed them, then a
    // gather, the scan and its merge (all return at once when every query certified), the merge
    // writing each result into the query's own output row.
    launch_gather_rows(d_qn, static_cast<uint32_t>(ds), d_fbq, d_fbn, n, d_qsub, s);
    ScanArgs fa;
    fa.tmap = &tmap_f32;
    fa.tmap_tile = &tmap_f32_176;
    fa.tmap_112 = &tmap_f32_112;
    fa.queries = d_qsub;
    fa.nq = n;
    fa.dq = static_cast<uint32_t>(ds);
    fa.rows = rows;
    fa.k = kcap;
    fa.ws_keys = d_ws;
    fa.status = d_status;
    fa.live = d_fbn;
    if ((e = launch_scan_fp32(fa, fb_plan, s)) != cudaSuccess) return cuda_error(e, "fallback scan launch");
    MergeArgs fm;
    fm.ws_keys = d_ws;
    fm.nq = n;
    fm.per_query = fb_per_query;
    fm.k = kcap;
    fm.out_stride = kcap;
    fm.idx_out = o_idx;
    fm.sim_out = o_sim;
    fm.count_out = o_cnt;
    fm.live = d_fbn;
    fm.out_rows = d_fbq;
    if ((st = merge_workspace(fb_per_query, n, kcap, fm, s))) return st;
    if ((e = launch_merge_topk(fm, s)) != cudaSuccess) return cuda_error(e, "fallback merge launch");
    last_tc_n = n;
    fbn_stream = s;
    fbn_pending = true;
    stats.kernel_launches += 6;
    stats.path = 6;
    stats.rerank_width = kp;
    stats.rows_scanned += rows * n;
    return NNDEX_OK;
}

// The device-side fallback's count into the statistics (waits for its stream once).
int CudaIndex::fetch_fallback_stats() {
    if (!fbn_pending) return NNDEX_OK;
    cudaMemcpyAsync(h_fbn, d_fbn, sizeof(uint32_t), cudaMemcpyDeviceToHost, fbn_stream);
    const cudaError_t e = cudaStreamSynchronize(fbn_stream);
    if (e != cudaSuccess) return cuda_error(e, "fallback count");
    fbn_pending = false;
    stats.fp32_fallback_queries = h_fbn[0];
    stats.certified = h_fbn[0] == 0 ? 1u : 0u;
    return NNDEX_OK;
}


int CudaIndex::tune_host(uint64_t n, uint64_t kcap, int mode, TunePlan* plan) {
    std::vector<TunePlan> cands = tune_candidates(n, kcap);
    const nndex_cuda_search_stats before = stats;
    const bool report = error_report;
    error_report = false;  // the timed runs record no score errors
    double best_ms = 0.0;
    int best = -1, last_err = NNDEX_OK;
    for (size_t c = 0; c < cands.size(); ++c) {
        double ms = 0.0;
        int cst = NNDEX_OK;
        for (int rep = 0; rep < 2 && cst == NNDEX_OK; ++rep) {
            forced_stride = cands[c].stride;
            forced_qb = cands[c].qb;
            const auto t0 = std::chrono::steady_clock::now();
            cst = enqueue_host_batch(n, kcap, mode, cands[c].path);
            const cudaError_t e = cudaStreamSynchronize(stream);
            if (cst == NNDEX_OK && e != cudaSuccess) cst = cuda_error(e, "search");
            if (cst == NNDEX_OK) cst = check_device_words();
            if (cst == NNDEX_OK && (cands[c].path == 2 || cands[c].path == 3))
                cst = finish_tc(static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt, stream);
            if (cst == NNDEX_OK && cands[c].path == 5)
                cst = ivf_finish_tc(*this, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt,
                                    stream);
            ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        forced_stride = 0;
        forced_qb = 0;
        if (cst != NNDEX_OK) {
            last_err = cst;
            continue;
        }
        if (best < 0 || ms < best_ms) {
            best = static_cast<int>(c);
            best_ms = ms;
        }
    }
    error_report = report;
    if (best < 0) return last_err;
    clear_error();
    TuneEntry ent;
    ent.plan = cands[best];
    ent.ms = best_ms;
    ent.candidates = static_cast<uint32_t>(cands.size());
    tune_cache[tune_key(n, kcap)] = ent;
    stats = before;
    stats.tuned = 1;
    stats.tune_candidates = ent.candidates;
    *plan = ent.plan;
    return NNDEX_OK;
}

// Enqueues one batch of the host-buffer search on `stream` (the queries already in h_q): status
// resets, upload, prep, the path's scan and merge, and the downloads into the pinned buffers.
int CudaIndex::enqueue_host_batch(uint64_t n, uint64_t kcap, int mode, int path) {
    int st;
    cudaMemsetAsync(d_err, 0xFF, sizeof(unsigned long long), stream);
    cudaMemsetAsync(d_status, 0, sizeof(uint32_t), stream);
    cudaMemcpyAsync(d_qraw, h_q, n * dims * sizeof(float), cudaMemcpyHostToDevice, stream);
    if ((st = enqueue_prep_queries(d_qraw, n, mode, path, stream))) return st;
    if (path == 4) {
        if ((st = ivf_search(*this, d_qn, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt,
                             stream)))
            return st;
    } else if (path == 5) {
        if ((st = ivf_search_tc(*this, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt,
                                stream)))
            return st;
    } else if (path == 1) {
        if ((st = enqueue_exact_fp32(d_qn, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap),
                                     static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt, stream)))
            return st;
    } else if (path == 6) {
        if ((st = enqueue_tf32(static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt, stream)))
            return st;
    } else {
        if ((st = enqueue_tc(path == 3, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt,
                             stream)))
            return st;
        if ((st = enqueue_tc_pass2(path == 3, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim,
                                   d_cnt, stream)))
            return st;
        // pass 2's counts come back with the results (finish_tc reads them once the batch is done)
        cudaMemcpyAsync(h_fbn, d_fbn, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    }
    if (error_report)
        serr_record(static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt, stream);
    cudaMemcpyAsync(h_res, d_res, res_bytes, cudaMemcpyDeviceToHost, stream);  // idx, sim, cnt
    cudaMemcpyAsync(h_flags, d_err, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream);  // err, status
    return NNDEX_OK;
}

// The batch through a CUDA graph when one is cached for this shape, capturing it when the same
// shape came in the previous call (its buffers are then allocated, so nothing allocates during
// the capture); otherwise directly. No path needs a host decision in the middle of its batch: the
// FP32 scan (1), the tensor-core scans (2, 3, 5: pass 2 and its compaction run on the device; the
// rare FP32 re-run of an overflowed collection follows the batch), the IVF list scan (4) and the
// TF32 candidate scan (6, its certificate's fallback on the device).
int CudaIndex::run_host_batch(uint64_t n, uint64_t kcap, int mode, int path) {
    const bool graphable = use_graphs && !scan_timing && !error_report && !sync_check_enabled() &&
                           path >= 1 && path <= 6 &&
                           !(graph_failed_paths & (1u << path));
    if (!graphable) return enqueue_host_batch(n, kcap, mode, path);
    const uint64_t epoch = alloc_epoch();
    const uint32_t np = static_cast<uint32_t>(ivf_scratch.nprobe);
    auto same = [&](const GraphEntry& g) {
        return g.path == path && g.mode == mode && g.n == n && g.kcap == kcap && g.nprobe == np;
    };
    for (size_t i = 0; i < graphs.size(); ++i) {
        if (!same(graphs[i])) continue;
        if (graphs[i].epoch != epoch) {
            cudaGraphExecDestroy(graphs[i].exec);
            graphs.erase(graphs.begin() + static_cast<long>(i));
            break;
        }
        const cudaError_t e = cudaGraphLaunch(graphs[i].exec, stream);
        if (e != cudaSuccess) return cuda_error(e, "graph launch");
        // the capture's statistics: counters added to this call's, the rest as captured
        const nndex_cuda_search_stats acc = stats;
        stats = graphs[i].stats;
        stats.kernel_launches += acc.kernel_launches;
        stats.rows_scanned += acc.rows_scanned;
        stats.second_pass_queries += acc.second_pass_queries;
        stats.fp32_fallback_queries += acc.fp32_fallback_queries;
        stats.ivf_rows_streamed = acc.ivf_rows_streamed;
        stats.ivf_rows_union = acc.ivf_rows_union;
        count_launch(static_cast<uint32_t>(graphs[i].launches));
        stats.graph = 2;
        if (path == 6) {  // the replayed fallback's count is read back with the statistics
            fbn_stream = stream;
            fbn_pending = true;
        }
        return NNDEX_OK;
    }
    if (!(same(graph_seen) && graph_seen.epoch == epoch)) {
        graph_seen = GraphEntry{path, mode, n, kcap, epoch, np};
        return enqueue_host_batch(n, kcap, mode, path);
    }
    // Second call of this shape with nothing reallocated in between: capture it.
    const nndex_cuda_search_stats before = stats;
    const uint64_t launches0 = kernel_launches_total();
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return enqueue_host_batch(n, kcap, mode, path);
    int st = enqueue_host_batch(n, kcap, mode, path);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (st == NNDEX_OK && e == cudaSuccess && alloc_epoch() == epoch)
        e = cudaGraphInstantiate(&exec, graph, 0);
    else if (e == cudaSuccess)
        e = cudaErrorStreamCaptureInvalidated;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();  // a failed capture leaves no sticky error
    if (e != cudaSuccess || !exec) {
        // run it the ordinary way; a path that cannot be captured is not tried again
        if (st == NNDEX_OK) graph_failed_paths |= 1u << path;
        stats = before;
        graph_seen = GraphEntry{};
        return enqueue_host_batch(n, kcap, mode, path);
    }
    GraphEntry g{path, mode, n, kcap, epoch, np};
    g.exec = exec;
    g.launches = kernel_launches_total() - launches0;
    g.stats = stats;  // counters as this batch's increments
    g.stats.kernel_launches -= before.kernel_launches;
    g.stats.rows_scanned -= before.rows_scanned;
    g.stats.second_pass_queries -= before.second_pass_queries;
    g.stats.fp32_fallback_queries -= before.fp32_fallback_queries;
    if (graphs.size() >= 8) {
        cudaGraphExecDestroy(graphs.front().exec);
        graphs.erase(graphs.begin());
    }
    graphs.push_back(g);
    if ((e = cudaGraphLaunch(exec, stream)) != cudaSuccess) return cuda_error(e, "graph launch");
    stats.graph = 1;
    return NNDEX_OK;
}

int CudaIndex::search_host(const float* queries, uint64_t nq, uint64_t k, int mode, uint64_t* idx_out,
                           float* sim_out, uint64_t* counts_out) {
    std::lock_guard<std::mutex> lock(mu);
    cudaSetDevice(device);
    stats = nndex_cuda_search_stats{};
    order_after_previous(stream);
    const uint64_t kcap = std::min<uint64_t>(k, rows);
    if (kcap > kMaxFusedK)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: k=%llu above the fused top-k limit %u",
                         (unsigned long long)kcap, kMaxFusedK);
    int st0;
    if (error_report && (st0 = serr_begin(nq, kcap, stream))) return st0;
    cudaEventRecord(ev0, stream);
    const uint64_t chunk = kMaxBatchChunk;
    for (uint64_t q0 = 0; q0 < nq; q0 += chunk) {
        const uint64_t n = std::min<uint64_t>(chunk, nq - q0);
        int st;
        if ((st = ensure_query_capacity(n))) return st;
        if ((st = ensure_result_capacity(n, kcap))) return st;
        std::memcpy(h_q, queries + q0 * dims, n * dims * sizeof(float));
        bool measure = false;
        TunePlan plan = plan_for(n, kcap, &measure);
        if (measure) {
            if ((st = tune_host(n, kcap, mode, &plan))) return st;
        } else if (autotune) {
            auto it = tune_cache.find(tune_key(n, kcap));
            if (it != tune_cache.end()) {
                stats.tuned = 2;
                stats.tune_candidates = it->second.candidates;
            }
        }
        const int path = plan.path;
        serr_off = q0;
        forced_stride = plan.stride;
        forced_qb = plan.qb;
        st = run_host_batch(n, kcap, mode, path);
        forced_stride = 0;
        forced_qb = 0;
        if (st) return st;
        cudaEventRecord(ev1, stream);  // before the wait: the device time ends with the last batch
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "search");
        if ((st = check_device_words())) return st;
        if (path == 2 || path == 3 || path == 5) {
            // pass 2 ran on the device; a query whose collection overflowed is re-run now
            st = path == 5 ? ivf_finish_tc(*this, static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim,
                                           d_cnt, stream)
                           : finish_tc(static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), d_idx, d_sim, d_cnt,
                                       stream);
            if (st) return st;
            if (stats.fp32_fallback_queries) {
                cudaMemcpyAsync(h_res, d_res, res_bytes, cudaMemcpyDeviceToHost, stream);
                if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_error(e, "search");
            }
        }
        if (path == 4) {
            stats.rows_scanned += ivf_scratch.h_probed[0];
            stats.ivf_rows_streamed += ivf_scratch.h_probed[1];
            stats.ivf_rows_union += ivf_scratch.h_probed[2];
        }
        std::memcpy(idx_out + q0 * kcap, h_idx, n * kcap * sizeof(uint64_t));
        std::memcpy(sim_out + q0 * kcap, h_sim, n * kcap * sizeof(float));
        if (counts_out)
            for (uint64_t i = 0; i < n; ++i) counts_out[q0 + i] = h_cnt[i];
    }
    mark_done(stream);
    float ms = 0.0f;
    if (nq) cudaEventElapsedTime(&ms, ev0, ev1);
    stats.device_ms = ms;
    return NNDEX_OK;
}

// One piece of a device-buffer search (≤ kMaxBatchChunk queries) on `path`: query prep, the path's
// scan and merge into the outputs. *synced is set when the path waited for the stream.
int CudaIndex::run_device_chunk(const float* dq, uint64_t n, uint64_t kcap, int path, uint64_t* oi, float* os,
                                uint32_t* oc, cudaStream_t s, bool* synced) {
    int st;
    if ((st = enqueue_prep_queries(dq, n, normalized ? 2 : 0, path, s))) return st;
    const uint32_t n32 = static_cast<uint32_t>(n), k32 = static_cast<uint32_t>(kcap);
    if (path == 4) return ivf_search(*this, d_qn, n32, k32, oi, os, oc, s);
    if (path == 5) {
        *synced = true;
        if ((st = ivf_search_tc(*this, n32, k32, oi, os, oc, s))) return st;
        h_flags[1] = 0;
        cudaMemcpyAsync(&h_flags[0], d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&h_flags[1], d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_error(e, "IVF search");
        if ((st = check_device_words())) return st;
        return ivf_finish_tc(*this, n32, k32, oi, os, oc, s);
    }
    if (path == 1) return enqueue_exact_fp32(d_qn, n32, k32, k32, oi, os, oc, s);
    // the certificates' fallbacks need the host: these paths synchronise
    *synced = true;
    if (path == 6) {
        *synced = false;  // the certificate's fallback runs on the device
        return enqueue_tf32(n32, k32, oi, os, oc, s);
    }
    if ((st = enqueue_tc(path == 3, n32, k32, oi, os, oc, s))) return st;
    if ((st = enqueue_tc_pass2(path == 3, n32, k32, oi, os, oc, s))) return st;
    cudaMemcpyAsync(h_fbn, d_fbn, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    h_flags[1] = 0;
    cudaMemcpyAsync(&h_flags[0], d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_flags[1], d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "search");
    if ((st = check_device_words())) return st;
    return finish_tc(n32, k32, oi, os, oc, s);
}

int CudaIndex::search_device(const float* d_queries, uint64_t nq, uint64_t k, uint64_t* d_idx_out,
                             float* d_sim_out, uint32_t* d_cnt_out, cudaStream_t s, int synchronize) {
    std::lock_guard<std::mutex> lock(mu);
    cudaSetDevice(device);
    stats = nndex_cuda_search_stats{};
    if (!s) s = cudaStreamLegacy;
    order_after_previous(s);
    const uint64_t kcap = std::min<uint64_t>(k, rows);
    int st;
    if ((st = ensure_query_capacity(std::min<uint64_t>(nq, kMaxBatchChunk)))) return st;
    if (error_report && (st = serr_begin(nq, kcap, s))) return st;
    cudaMemsetAsync(d_err, 0xFF, sizeof(unsigned long long), s);
    cudaMemsetAsync(d_status, 0, sizeof(uint32_t), s);
    bool synced = false;
    for (uint64_t q0 = 0; q0 < nq; q0 += kMaxBatchChunk) {
        const uint64_t n = std::min<uint64_t>(kMaxBatchChunk, nq - q0);
        uint64_t* oi = d_idx_out + q0 * kcap;
        float* os = d_sim_out + q0 * kcap;
        uint32_t* oc = d_cnt_out ? d_cnt_out + q0 : nullptr;
        const float* dq = d_queries + q0 * dims;
        bool measure = false;
        TunePlan plan = plan_for(n, kcap, &measure);
        if (measure) {
            // the first batch of this shape: time every candidate plan on it, keep the fastest
            std::vector<TunePlan> cands = tune_candidates(n, kcap);
            const nndex_cuda_search_stats before = stats;
            double best_ms = 0.0;
            int best = -1, last_err = NNDEX_OK;
            for (size_t c = 0; c < cands.size(); ++c) {
                double ms = 0.0;
                int cst = NNDEX_OK;
                for (int rep = 0; rep < 2 && cst == NNDEX_OK; ++rep) {
                    forced_stride = cands[c].stride;
                    forced_qb = cands[c].qb;
                    bool sy = false;
                    const auto t0 = std::chrono::steady_clock::now();
                    cst = run_device_chunk(dq, n, kcap, cands[c].path, oi, os, oc, s, &sy);
                    const cudaError_t e = cudaStreamSynchronize(s);
                    if (cst == NNDEX_OK && e != cudaSuccess) cst = cuda_error(e, "search");
                    ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                }
                forced_stride = 0;
                forced_qb = 0;
                if (cst != NNDEX_OK) {
                    last_err = cst;
                    continue;
                }
                if (best < 0 || ms < best_ms) {
                    best = static_cast<int>(c);
                    best_ms = ms;
                }
            }
            if (best < 0) return last_err;
            clear_error();
            TuneEntry ent;
            ent.plan = cands[best];
            ent.ms = best_ms;
            ent.candidates = static_cast<uint32_t>(cands.size());
            tune_cache[tune_key(n, kcap)] = ent;
            stats = before;
            stats.tuned = 1;
            stats.tune_candidates = ent.candidates;
            plan = ent.plan;
            synced = true;
        } else if (autotune) {
            auto it = tune_cache.find(tune_key(n, kcap));
            if (it != tune_cache.end()) {
                stats.tuned = 2;
                stats.tune_candidates = it->second.candidates;
            }
        }
        forced_stride = plan.stride;
        forced_qb = plan.qb;
        st = run_device_chunk(dq, n, kcap, plan.path, oi, os, oc, s, &synced);
        forced_stride = 0;
        forced_qb = 0;
        if (st) return st;
        if (error_report) {
            serr_off = q0;
            serr_record(static_cast<uint32_t>(n), static_cast<uint32_t>(kcap), oi, os, oc, s);
        }
    }
    if (synchronize || synced) {
        h_flags[1] = 0;
        cudaMemcpyAsync(&h_flags[0], d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&h_flags[1], d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        mark_done(s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_error(e, "search");
        if (stats.path == 4) {
            stats.rows_scanned = ivf_scratch.h_probed[0];
            stats.ivf_rows_streamed = ivf_scratch.h_probed[1];
            stats.ivf_rows_union = ivf_scratch.h_probed[2];
        }
        return check_device_words();
    }
    mark_done(s);
    return NNDEX_OK;
}

// Score-error report: buffers for the call's nq × kcap results and a cleared accumulator.
int CudaIndex::serr_begin(uint64_t nq, uint64_t kcap, cudaStream_t s) {
    int st;
    if ((st = grow_device(d_serr, cap_serr, nq * kcap, "score-error buffer"))) return st;
    if (!d_serr_acc) {
        cudaError_t e;
        if ((e = cudaMalloc(&d_serr_acc, 3 * sizeof(unsigned long long))) != cudaSuccess ||
            (e = cudaMallocHost(&h_serr_acc, 3 * sizeof(unsigned long long))) != cudaSuccess)
            return cuda_error(e, "score-error buffer");
    }
    cudaMemsetAsync(d_serr_acc, 0, 3 * sizeof(unsigned long long), s);
    serr_nq = nq;
    serr_k = kcap;
    serr_off = 0;
    serr_stream = s;
    serr_pending = true;
    stats.score_errors = 1;
    return NNDEX_OK;
}

// The errors of one piece of the call (its first query at serr_off; queries normalised in d_qn).
void CudaIndex::serr_record(uint32_t n, uint32_t kcap, const uint64_t* idx, const float* sim, const uint32_t* cnt,
                            cudaStream_t s) {
    launch_score_errors(d_base, ds, d_qn, n, kcap, idx, sim, cnt, d_serr + serr_off * kcap, d_serr_acc, s);
    stats.kernel_launches += 1;
}

// Max and mean error into the statistics, once per call (waits for the call's stream).
int CudaIndex::serr_fetch_stats() {
    if (!serr_pending) return NNDEX_OK;
    cudaMemcpyAsync(h_serr_acc, d_serr_acc, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, serr_stream);
    const cudaError_t e = cudaStreamSynchronize(serr_stream);
    if (e != cudaSuccess) return cuda_error(e, "score errors");
    serr_pending = false;
    double mx, sum;
    std::memcpy(&mx, &h_serr_acc[0], sizeof(double));
    std::memcpy(&sum, &h_serr_acc[1], sizeof(double));
    stats.max_score_error = mx;
    stats.mean_score_error = h_serr_acc[2] ? sum / static_cast<double>(h_serr_acc[2]) : 0.0;
    return NNDEX_OK;
}

// The index's scratch buffers are shared by every call: work enqueued on one stream must not
// overlap work of an earlier call on another stream.
void CudaIndex::order_after_previous(cudaStream_t s) {
    if (done_ev && done_stream && done_stream != s) cudaStreamWaitEvent(s, done_ev, 0);
}
void CudaIndex::mark_done(cudaStream_t s) {
    if (!done_ev) cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming);
    cudaEventRecord(done_ev, s);
    done_stream = s;
}

int CudaIndex::stream_status() {
    std::lock_guard<std::mutex> lock(mu);
    cudaSetDevice(device);
    h_flags[1] = 0;
    cudaStreamSynchronize(stream);
    cudaMemcpy(&h_flags[0], d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost);
    cudaMemcpy(&h_flags[1], d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    return check_device_words();
}

// ---- construction ----------------------------------------------------------------------------

static int select_device(int32_t requested, int& device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
    int d = requested < 0 ? 0 : requested;
    if (d >= n)
        return set_error(NNDEX_ERR_DEVICE_INDEX, "gpu device index %d is out of range (found %d adapter(s))", d, n);
    device = d;
    return NNDEX_OK;
}

// Construction in three steps (create_index below, and the streaming builder in builder.cu):
// index_begin allocates the device copies for rows × dims; index_prep_rows runs K1 (validate,
// normalise, pad, low-precision copies) over raw rows already on the device; index_finish checks
// the error word and completes the index (residual bounds, tensor maps, the IVF).
int index_begin(uint64_t rows, uint64_t dims, uint32_t flags, const nndex_cuda_opts* opts, CudaIndex** out) {
    *out = nullptr;
    if (rows >= (1ull << 31))
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: rows=%llu above the 2^31-1 row limit",
                         (unsigned long long)rows);
    const uint64_t dp = (dims + 7) / 8 * 8;
    if (dp > NNDEX_MAX_DIMS)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: dims=%llu above the %u limit",
                         (unsigned long long)dims, NNDEX_MAX_DIMS);
    nndex_cuda_opts o{};
    o.device = -1;
    if (opts) o = *opts;
    int device = 0;
    int st = select_device(o.device, device);
    if (st) return st;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    // The no-allocation entry point's array is bound here, on the index's device: with lazy module
    // loading its memory is taken when its address is first looked up.
    if ((st = noalloc_bind(device))) return st;

    CudaIndex* ix = new (std::nothrow) CudaIndex();
    if (!ix) return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: host allocation failed");
    ix->device = device;
    ix->rows = rows;
    ix->dims = dims;
    ix->dp = dp;
    ix->ds = (dims + 31) / 32 * 32;
    ix->rows_alloc = (rows + 255) / 256 * 256;  // whole 256-row tensor-core tiles
    ix->flags = flags;
    ix->precision = o.precision;
    ix->rerank_width = o.rerank_width;
    ix->normalized = (flags & NNDEX_FLAG_NORMALIZED) != 0;
    ix->approx = (flags & NNDEX_FLAG_APPROX) != 0;
    ix->opts = o;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ix->sm_count = prop.multiProcessorCount;
    ix->smem_optin = prop.sharedMemPerBlockOptin;
    auto fail = [&](int code) {
        delete ix;
        return code;
    };
    if ((e = cudaStreamCreateWithFlags(&ix->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(cuda_error(e, "cudaStreamCreate"));
    cudaEventCreate(&ix->ev0);
    cudaEventCreate(&ix->ev1);
    if ((e = cudaMalloc(&ix->d_err, 2 * sizeof(unsigned long long))) != cudaSuccess) return fail(cuda_error(e, "alloc"));
    ix->d_status = reinterpret_cast<uint32_t*>(ix->d_err + 1);
    if ((e = cudaMallocHost(&ix->h_flags, 2 * sizeof(uint64_t))) != cudaSuccess) return fail(cuda_error(e, "alloc"));
    const size_t base_bytes = ix->rows_alloc * ix->ds * sizeof(float);
    if ((e = cudaMalloc(&ix->d_base, base_bytes)) != cudaSuccess) return fail(cuda_error(e, "base allocation"));
    cudaMemsetAsync(ix->d_base + rows * ix->ds, 0, (ix->rows_alloc - rows) * ix->ds * sizeof(float), ix->stream);
    cudaMemsetAsync(ix->d_err, 0xFF, sizeof(unsigned long long), ix->stream);
    cudaMemsetAsync(ix->d_status, 0, sizeof(uint32_t), ix->stream);
    // Low-precision scoring copies (K1 writes them in the same pass) and their residual norms.
    if (flags & NNDEX_FLAG_BF16) {
        ix->kb16 = (dims + 63) / 64 * 64;
        if ((e = cudaMalloc(&ix->d_base_bf16, ix->rows_alloc * ix->kb16 * 2)) != cudaSuccess ||
            (e = cudaMalloc(&ix->d_res16, rows * sizeof(float))) != cudaSuccess)
            return fail(cuda_error(e, "BF16 copy allocation"));
        cudaMemsetAsync(ix->d_base_bf16, 0, ix->rows_alloc * ix->kb16 * 2, ix->stream);
    }
    if (flags & NNDEX_FLAG_FP8) {
        ix->kf8 = (dims + 127) / 128 * 128;
        if ((e = cudaMalloc(&ix->d_base_fp8, ix->rows_alloc * ix->kf8)) != cudaSuccess ||
            (e = cudaMalloc(&ix->d_row_scale, ix->rows_alloc * sizeof(float))) != cudaSuccess ||
            (e = cudaMalloc(&ix->d_res8, rows * sizeof(float))) != cudaSuccess)
            return fail(cuda_error(e, "FP8 copy allocation"));
        cudaMemsetAsync(ix->d_base_fp8, 0, ix->rows_alloc * ix->kf8, ix->stream);
        cudaMemsetAsync(ix->d_row_scale, 0, ix->rows_alloc * sizeof(float), ix->stream);
    }
    *out = ix;
    return NNDEX_OK;
}

void index_prep_rows(CudaIndex* ix, const float* d_src, uint64_t row0, uint64_t n) {
    PrepArgs p;
    p.src = d_src;
    p.rows = n;
    p.dims = static_cast<uint32_t>(ix->dims);
    p.row_base = row0;
    p.out = ix->d_base + row0 * ix->ds;
    p.out_stride = static_cast<uint32_t>(ix->ds);
    p.mode = ix->normalized ? 2 : 0;
    p.err = ix->d_err;
    p.sm_count = ix->sm_count;
    if (ix->d_base_bf16) {
        p.out_bf16 = ix->d_base_bf16 + row0 * ix->kb16;
        p.bf16_stride = static_cast<uint32_t>(ix->kb16);
        p.resid_bf16 = ix->d_res16 + row0;
    }
    if (ix->d_base_fp8) {
        p.out_fp8 = ix->d_base_fp8 + row0 * ix->kf8;
        p.fp8_stride = static_cast<uint32_t>(ix->kf8);
        p.fp8_scale = ix->d_row_scale + row0;
        p.resid_fp8 = ix->d_res8 + row0;
    }
    launch_prep_rows(p, ix->stream);
}

int index_finish(CudaIndex* ix) {
    auto fail = [&](int code) {
        delete ix;
        return code;
    };
    cudaError_t e;
    cudaMemcpyAsync(&ix->h_flags[0], ix->d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost, ix->stream);
    if ((e = cudaStreamSynchronize(ix->stream)) != cudaSuccess) return fail(cuda_error(e, "upload"));
    if (ix->h_flags[0] != ~0ull) return fail(err_code(static_cast<int>(ix->h_flags[0] & 0xFF)));
    if (ix->d_res16 || ix->d_res8) {
        // ε of the certificate: the largest residual norm ‖x − x̂‖ over the rows.
        unsigned int* d_max = nullptr;
        if ((e = cudaMalloc(&d_max, 2 * sizeof(unsigned int))) != cudaSuccess) return fail(cuda_error(e, "alloc"));
        cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned int), ix->stream);
        if (ix->d_res16) launch_max_reduce(ix->d_res16, ix->rows, d_max, ix->stream);
        if (ix->d_res8) launch_max_reduce(ix->d_res8, ix->rows, d_max + 1, ix->stream);
        unsigned int hm[2] = {0, 0};
        cudaMemcpyAsync(hm, d_max, sizeof(hm), cudaMemcpyDeviceToHost, ix->stream);
        e = cudaStreamSynchronize(ix->stream);
        cudaFree(d_max);
        if (e != cudaSuccess) return fail(cuda_error(e, "residual reduction"));
        std::memcpy(&ix->eps_bf16, &hm[0], 4);
        std::memcpy(&ix->eps_fp8, &hm[1], 4);
    }
    if (!encode_tmap_2d(&ix->tmap_f32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ix->d_base, ix->ds, ix->rows_alloc,
                        ix->ds * sizeof(float), 32, 128, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_tmap_2d(&ix->tmap_f32_176, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ix->d_base, ix->ds, ix->rows_alloc,
                        ix->ds * sizeof(float), 32, 176, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_tmap_2d(&ix->tmap_f32_112, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ix->d_base, ix->ds, ix->rows_alloc,
                        ix->ds * sizeof(float), 32, 112, CU_TENSOR_MAP_SWIZZLE_128B))
        return fail(set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed"));
    if (ix->d_base_bf16 &&
        (!encode_tmap_2d(&ix->tmap_bf16, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ix->d_base_bf16, ix->kb16,
                         ix->rows_alloc, ix->kb16 * 2, 64, 256, CU_TENSOR_MAP_SWIZZLE_128B) ||
         !encode_tmap_2d(&ix->tmap_bf16_h, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ix->d_base_bf16, ix->kb16,
                         ix->rows_alloc, ix->kb16 * 2, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B)))
        return fail(set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed (BF16)"));
    if (ix->d_base_fp8 &&
        (!encode_tmap_2d(&ix->tmap_fp8, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ix->d_base_fp8, ix->kf8, ix->rows_alloc,
                         ix->kf8, 128, 256, CU_TENSOR_MAP_SWIZZLE_128B) ||
         !encode_tmap_2d(&ix->tmap_fp8_h, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ix->d_base_fp8, ix->kf8, ix->rows_alloc,
                         ix->kf8, 128, 128, CU_TENSOR_MAP_SWIZZLE_128B)))
        return fail(set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed (FP8)"));
    if (ix->d_row_scale) {
        // FP8 scan: the scale extremes of each 256-row tile (its epilogue's per-tile cut)
        if ((e = cudaMalloc(&ix->d_tile_scale, ix->rows_alloc / 256 * sizeof(float2))) != cudaSuccess)
            return fail(cuda_error(e, "FP8 tile scales"));
        launch_tile_scale(ix->d_row_scale, ix->rows, ix->rows_alloc / 256, ix->d_tile_scale, ix->stream);
    }
    // Row norms of K12's bound (8 bytes per row, one pass over the base). Without them (no memory)
    // small batches take the FP32 scan.
    if (cudaMalloc(&ix->d_tfnorm, ix->rows * sizeof(float2)) == cudaSuccess) {
        if ((e = launch_tf32_row_norms(ix->d_base, ix->rows, static_cast<uint32_t>(ix->ds), ix->d_tfnorm,
                                       static_cast<uint32_t>(ix->sm_count), ix->stream)) != cudaSuccess)
            return fail(cuda_error(e, "row norms launch"));
    } else {
        ix->d_tfnorm = nullptr;
        cudaGetLastError();
    }
    if (ix->approx) {
        // src/approx.rs:46-100, built once at construction instead of on the first approx search.
        const int st = ivf_build(*ix);
        if (st != NNDEX_OK) return fail(st);
    }
    return NNDEX_OK;
}

int create_index(const float* matrix, bool on_device, uint64_t n_values, uint64_t rows, uint64_t dims,
                 uint32_t flags, const nndex_cuda_opts* opts, CudaIndex** out) {
    if (!out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null output handle");
    *out = nullptr;
    if (!shape_ok(n_values, rows, dims)) return err_shape(rows, dims, n_values);
    if (!matrix) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null matrix");
    CudaIndex* ix = nullptr;
    int st = index_begin(rows, dims, flags, opts, &ix);
    if (st) return st;
    cudaError_t e = cudaSuccess;
    // K1: upload in chunks (≈256 MB of raw rows each), validate + normalise + pad on the device.
    if (on_device) {
        // The caller may still be writing the matrix on any stream: wait for the device first.
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
            delete ix;
            return cuda_error(e, "cudaDeviceSynchronize");
        }
        index_prep_rows(ix, matrix, 0, rows);
    } else {
        uint64_t chunk_rows = std::max<uint64_t>(1, (256ull << 20) / (dims * sizeof(float)));
        chunk_rows = std::min(chunk_rows, rows);
        float* d_raw[2] = {nullptr, nullptr};
        cudaEvent_t done[2];
        for (int b = 0; b < 2; ++b) {
            if ((e = cudaMalloc(&d_raw[b], chunk_rows * dims * sizeof(float))) != cudaSuccess) {
                cudaFree(d_raw[0]);
                delete ix;
                return cuda_error(e, "upload staging");
            }
            cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming);
        }
        int b = 0;
        for (uint64_t r0 = 0; r0 < rows; r0 += chunk_rows, b ^= 1) {
            const uint64_t n = std::min(chunk_rows, rows - r0);
            cudaEventSynchronize(done[b]);
            e = cudaMemcpyAsync(d_raw[b], matrix + r0 * dims, n * dims * sizeof(float), cudaMemcpyHostToDevice,
                                ix->stream);
            if (e != cudaSuccess) break;
            index_prep_rows(ix, d_raw[b], r0, n);
            cudaEventRecord(done[b], ix->stream);
        }
        cudaStreamSynchronize(ix->stream);
        for (int i = 0; i < 2; ++i) {
            cudaFree(d_raw[i]);
            cudaEventDestroy(done[i]);
        }
        if (e != cudaSuccess) {
            delete ix;
            return cuda_error(e, "upload");
        }
    }
    if ((st = index_finish(ix))) return st;
    *out = ix;
    return NNDEX_OK;
}

// A second handle on the same device-resident index: it shares the read-only data (base copies,
// tensor maps, the IVF) and owns its stream, status words and per-search scratch, so several can
// search concurrently (server slots).
int make_view(const CudaIndex& src, CudaIndex** out) {
    *out = nullptr;
    cudaSetDevice(src.device);
    CudaIndex* v = new (std::nothrow) CudaIndex();
    if (!v) return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: host allocation failed");
    v->owns_base = false;
    v->device = src.device;
    v->sm_count = src.sm_count;
    v->smem_optin = src.smem_optin;
    v->rows = src.rows;
    v->rows_alloc = src.rows_alloc;
    v->dims = src.dims;
    v->dp = src.dp;
    v->ds = src.ds;
    v->flags = src.flags;
    v->normalized = src.normalized;
    v->approx = src.approx;
    v->opts = src.opts;
    v->d_base = src.d_base;
    v->tmap_f32 = src.tmap_f32;
    v->tmap_f32_176 = src.tmap_f32_176;
    v->tmap_f32_112 = src.tmap_f32_112;
    v->precision = src.precision;
    v->kb16 = src.kb16;
    v->kf8 = src.kf8;
    v->d_base_bf16 = src.d_base_bf16;
    v->d_base_fp8 = src.d_base_fp8;
    v->d_row_scale = src.d_row_scale;
    v->d_tile_scale = src.d_tile_scale;
    v->eps_bf16 = src.eps_bf16;
    v->eps_fp8 = src.eps_fp8;
    v->d_res16 = src.d_res16;
    v->d_res8 = src.d_res8;
    v->d_tfnorm = src.d_tfnorm;
    v->tmap_bf16 = src.tmap_bf16;
    v->tmap_fp8 = src.tmap_fp8;
    v->tmap_bf16_h = src.tmap_bf16_h;
    v->tmap_fp8_h = src.tmap_fp8_h;
    v->rerank_width = src.rerank_width;
    v->tc_sample_stride = src.tc_sample_stride;
    // a view (a serving slot) never stops a batch to time plans: the source's measured plans, else
    // the rules
    v->tune_cache = src.tune_cache;
    v->autotune = src.autotune ? 2 : 0;
    v->ivf = src.ivf;
    v->ivf_scratch.nprobe = src.ivf_scratch.nprobe;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&v->ev0)) != cudaSuccess || (e = cudaEventCreate(&v->ev1)) != cudaSuccess ||
        (e = cudaMalloc(&v->d_err, 2 * sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMallocHost(&v->h_flags, 2 * sizeof(uint64_t))) != cudaSuccess) {
        delete v;
        return cuda_error(e, "index view");
    }
    v->d_status = reinterpret_cast<uint32_t*>(v->d_err + 1);
    cudaMemsetAsync(v->d_err, 0xFF, sizeof(unsigned long long), v->stream);
    cudaMemsetAsync(v->d_status, 0, sizeof(uint32_t), v->stream);
    cudaStreamSynchronize(v->stream);
    *out = v;
    return NNDEX_OK;
}

int fill_devinfo(int device, nndex_cuda_devinfo* out) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
    std::memset(out, 0, sizeof(*out));
    out->index = static_cast<uint64_t>(device);
    std::snprintf(out->name, sizeof(out->name), "%s", prop.name);
    std::snprintf(out->driver, sizeof(out->driver), "NVIDIA");
    int drv = 0, rt = 0;
    cudaDriverGetVersion(&drv);
    cudaRuntimeGetVersion(&rt);
    std::snprintf(out->driver_info, sizeof(out->driver_info), "CUDA driver %d.%d, runtime %d.%d", drv / 1000,
                  (drv % 1000) / 10, rt / 1000, (rt % 1000) / 10);
    std::snprintf(out->backend, sizeof(out->backend), "Cuda");
    std::snprintf(out->device_type, sizeof(out->device_type), prop.integrated ? "IntegratedGpu" : "DiscreteGpu");
    out->sm_count = prop.multiProcessorCount;
    out->cc_major = prop.major;
    out->cc_minor = prop.minor;
    out->hbm_bytes = prop.totalGlobalMem;
    out->l2_bytes = prop.l2CacheSize;
    return NNDEX_OK;
}

uint64_t launches() { return g_launches.load(); }

}  // namespace nndex

// =============================================================================================
// C ABI
// =============================================================================================
using namespace nndex;

extern "C" {

const char* nndex_cuda_last_error(void) { return last_error(); }

uint64_t nndex_cuda_kernel_launch_count(void) { return launches(); }

int nndex_cuda_set_scan_timing(nndex_cuda_index* index, int enable) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    std::lock_guard<std::mutex> lock(index->impl->mu);
    index->impl->scan_timing = enable != 0;
    return NNDEX_OK;
}

int nndex_cuda_scan_timing(nndex_cuda_index* index, double* total_ms, uint64_t* launches_out) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    double sum = 0.0;
    for (size_t i = 0; i < ix->scan_events_used; ++i) {
        cudaError_t e = cudaEventSynchronize(ix->scan_events[i].second);
        if (e != cudaSuccess) return cuda_error(e, "scan timing");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ix->scan_events[i].first, ix->scan_events[i].second);
        sum += ms;
    }
    if (total_ms) *total_ms = sum;
    if (launches_out) *launches_out = ix->scan_events_used;
    ix->scan_events_used = 0;
    return NNDEX_OK;
}

int nndex_cuda_list_devices(nndex_cuda_devinfo* out, uint32_t capacity, uint32_t* count) {
    clear_error();
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) n = 0;
    else if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
    if (count) *count = static_cast<uint32_t>(n);
    for (int d = 0; d < n && static_cast<uint32_t>(d) < capacity && out; ++d) {
        int st = fill_devinfo(d, &out[d]);
        if (st) return st;
    }
    return NNDEX_OK;
}

int nndex_cuda_info(const nndex_cuda_index* index, nndex_cuda_devinfo* out) {
    clear_error();
    if (!index || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    return fill_devinfo(index->impl->device, out);
}

int nndex_cuda_create(const float* host_matrix, uint64_t n_values, uint64_t rows, uint64_t dims, uint32_t flags,
                      const nndex_cuda_opts* opts, nndex_cuda_index** out) {
    clear_error();
    if (!out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null output handle");
    CudaIndex* impl = nullptr;
    int st = create_index(host_matrix, false, n_values, rows, dims, flags, opts, &impl);
    if (st) return st;
    *out = new nndex_cuda_index{impl};
    return NNDEX_OK;
}

int nndex_cuda_create_from_device(const float* device_matrix, uint64_t n_values, uint64_t rows, uint64_t dims,
                                  uint32_t flags, const nndex_cuda_opts* opts, nndex_cuda_index** out) {
    clear_error();
    if (!out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null output handle");
    CudaIndex* impl = nullptr;
    int st = create_index(device_matrix, true, n_values, rows, dims, flags, opts, &impl);
    if (st) return st;
    *out = new nndex_cuda_index{impl};
    return NNDEX_OK;
}

void nndex_cuda_destroy(nndex_cuda_index* index) {
    if (!index) return;
    delete index->impl;
    delete index;
}

int nndex_cuda_rows(const nndex_cuda_index* index, uint64_t* rows, uint64_t* dims, uint64_t* padded_dims) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    if (rows) *rows = index->impl->rows;
    if (dims) *dims = index->impl->dims;
    if (padded_dims) *padded_dims = index->impl->dp;
    return NNDEX_OK;
}

int nndex_cuda_search(nndex_cuda_index* index, const float* host_query, uint64_t query_len, uint64_t k,
                      uint64_t* idx_out, float* sim_out, uint64_t* count_out) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    // src/lib.rs:336-344: k == 0 first, then the dimensionality.
    if (k == 0) return err_topk();
    if (query_len != ix->dims) return err_query_dims(ix->dims, query_len);
    if (!host_query || !idx_out || !sim_out)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null buffer");
    uint64_t cnt = 0;
    int st = ix->search_host(host_query, 1, k, ix->normalized ? 2 : 1, idx_out, sim_out, &cnt);
    if (st) return st;
    if (count_out) *count_out = cnt;
    return NNDEX_OK;
}

int nndex_cuda_search_batch(nndex_cuda_index* index, const float* host_queries, uint64_t n_values,
                            uint64_t query_rows, uint64_t k, uint64_t* idx_out, float* sim_out,
                            uint64_t* counts_out) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    // src/lib.rs:378-381: the shape first, then k == 0.
    if (!shape_ok(n_values, query_rows, ix->dims)) return err_shape(query_rows, ix->dims, n_values);
    if (k == 0) return err_topk();
    if (!host_queries || !idx_out || !sim_out)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null buffer");
    return ix->search_host(host_queries, query_rows, k, ix->normalized ? 2 : 0, idx_out, sim_out, counts_out);
}

int nndex_cuda_search_batch_device(nndex_cuda_index* index, const float* dev_queries, uint64_t query_rows,
                                   uint64_t query_dims, uint64_t k, uint64_t* dev_idx_out, float* dev_sim_out,
                                   uint32_t* dev_counts_out, void* stream, int synchronize) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    if (query_rows == 0 || query_dims != ix->dims) return err_shape(query_rows, ix->dims, query_rows * query_dims);
    if (k == 0) return err_topk();
    if (!dev_queries || !dev_idx_out || !dev_sim_out)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null buffer");
    if (std::min<uint64_t>(k, ix->rows) > kMaxFusedK)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: k above the fused top-k limit %u",
                         kMaxFusedK);
    return ix->search_device(dev_queries, query_rows, k, dev_idx_out, dev_sim_out, dev_counts_out,
                             static_cast<cudaStream_t>(stream), synchronize);
}

int nndex_cuda_set_precision(nndex_cuda_index* index, uint32_t precision, uint32_t rerank_width) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    if (precision > NNDEX_PRECISION_FP8)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: unknown precision %u", precision);
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    if ((precision == NNDEX_PRECISION_BF16 && !ix->d_base_bf16) || (precision == NNDEX_PRECISION_FP8 && !ix->d_base_fp8))
        return set_error(NNDEX_ERR_INVALID_ARGUMENT,
                         "cuda execution error: the index keeps no %s copy (create it with NNDEX_FLAG_%s)",
                         precision == NNDEX_PRECISION_BF16 ? "BF16" : "FP8",
                         precision == NNDEX_PRECISION_BF16 ? "BF16" : "FP8");
    ix->precision = precision;
    ix->drop_graphs();
    ix->rerank_width = rerank_width;
    return NNDEX_OK;
}

int nndex_cuda_last_candidates(nndex_cuda_index* index, uint64_t query_rows, uint64_t* idx_out, float* approx_out,
                               uint64_t capacity, uint32_t* kprime, float* eps_rows, uint32_t* certified_out) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    const uint32_t kp = ix->stats.rerank_width;
    if (kprime) *kprime = kp;
    if (eps_rows)
        *eps_rows = ix->stats.path == 3 ? ix->eps_fp8 : ix->stats.path == 6 ? ix->tf32_eps() : ix->eps_bf16;
    if (kp == 0 || !ix->d_cand_idx) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: no low-precision search yet");
    if (ix->stats.path == 5)
        return set_error(NNDEX_ERR_UNSUPPORTED,
                         "cuda execution error: the IVF list scan's candidates are list positions, not exported");
    const uint64_t n = query_rows * kp;
    if (n > capacity || n > ix->cap_cand_idx)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: candidate buffer too small");
    cudaError_t e = cudaDeviceSynchronize();  // the search may have run on any stream
    if (e == cudaSuccess && idx_out) e = cudaMemcpy(idx_out, ix->d_cand_idx, n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && approx_out) e = cudaMemcpy(approx_out, ix->d_cand_sim, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && certified_out) {
        if (query_rows > ix->last_tc_n)
            return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: more rows than the last batch");
        e = cudaMemcpy(certified_out, ix->d_cert, query_rows * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    }
    if (e != cudaSuccess) return cuda_error(e, "candidates");
    return NNDEX_OK;
}

int nndex_cuda_stream_status(nndex_cuda_index* index) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    return index->impl->stream_status();
}

int nndex_cuda_last_search_stats(const nndex_cuda_index* index, nndex_cuda_search_stats* out) {
    clear_error();
    if (!index || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    if (ix->serr_pending || ix->fbn_pending) {
        cudaSetDevice(ix->device);
        int st = ix->serr_fetch_stats();
        if (!st) st = ix->fetch_fallback_stats();
        if (st) return st;
    }
    *out = ix->stats;
    return NNDEX_OK;
}

int nndex_cuda_set_error_report(nndex_cuda_index* index, int enable) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    cudaStreamSynchronize(ix->stream);
    ix->error_report = enable != 0;
    ix->drop_graphs();
    return NNDEX_OK;
}

int nndex_cuda_last_score_errors(nndex_cuda_index* index, uint64_t query_rows, uint64_t k, double* errors_out) {
    clear_error();
    if (!index || !errors_out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    const uint64_t kcap = std::min<uint64_t>(k, ix->rows);
    if (!ix->stats.score_errors || !ix->d_serr)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: the last search recorded no score errors "
                                                     "(nndex_cuda_set_error_report)");
    if (query_rows != ix->serr_nq || kcap != ix->serr_k)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT,
                         "cuda execution error: the last search had %llu queries at k=%llu, not %llu at k=%llu",
                         (unsigned long long)ix->serr_nq, (unsigned long long)ix->serr_k,
                         (unsigned long long)query_rows, (unsigned long long)kcap);
    cudaSetDevice(ix->device);
    cudaError_t e = cudaStreamSynchronize(ix->serr_stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(errors_out, ix->d_serr, query_rows * kcap * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "score errors");
    return NNDEX_OK;
}

int nndex_cuda_ivf_layout(nndex_cuda_index* index, uint64_t* nlist_out, float* centroids, uint64_t* offsets,
                          uint64_t* original_indices, uint64_t* init_rows) {
    clear_error();
    if (!index || !nlist_out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    *nlist_out = 0;
    if (!ix->ivf) return NNDEX_OK;
    const IvfIndex& v = *ix->ivf;
    *nlist_out = v.nlist;
    cudaSetDevice(ix->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && centroids)
        e = cudaMemcpy2D(centroids, ix->dp * sizeof(float), v.d_centroids, ix->ds * sizeof(float), ix->dp * sizeof(float),
                         v.nlist, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && original_indices) {
        std::vector<uint32_t> m(ix->rows);
        e = cudaMemcpy(m.data(), v.d_row_map, ix->rows * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        for (uint64_t i = 0; i < ix->rows; ++i) original_indices[i] = m[i];
    }
    if (e != cudaSuccess) return cuda_error(e, "IVF layout copy");
    if (offsets) std::copy(v.h_offsets.begin(), v.h_offsets.end(), offsets);
    if (init_rows) std::copy(v.h_init_rows.begin(), v.h_init_rows.end(), init_rows);
    return NNDEX_OK;
}

int nndex_cuda_ivf_restore(nndex_cuda_index* index, uint64_t nlist, const float* centroids, const uint64_t* offsets,
                           const uint64_t* original_indices, const uint64_t* init_rows) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    if (!ix->owns_base)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: cannot restore an IVF into a view");
    cudaSetDevice(ix->device);
    cudaError_t e = cudaDeviceSynchronize();  // searches in flight on any stream read the old IVF
    if (e != cudaSuccess) return cuda_error(e, "IVF restore");
    ix->drop_graphs();
    const int st = ivf_restore(*ix, nlist, centroids, offsets, original_indices, init_rows);
    if (st == NNDEX_OK) ix->approx = true;
    return st;
}

int nndex_cuda_base_checksum(nndex_cuda_index* index, uint64_t* checksum) {
    clear_error();
    if (!index || !checksum) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(e, "checksum");
    return base_checksum(*ix, checksum);
}

int nndex_cuda_set_graphs(nndex_cuda_index* index, int enable) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    cudaStreamSynchronize(ix->stream);
    ix->use_graphs = enable != 0;
    ix->drop_graphs();
    return NNDEX_OK;
}

int nndex_cuda_set_nprobe(nndex_cuda_index* index, uint32_t nprobe) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    ix->opts.nprobe = nprobe;
    ix->ivf_scratch.nprobe = nprobe;
    ix->drop_graphs();
    return NNDEX_OK;
}

int nndex_cuda_ivf_stats_get(const nndex_cuda_index* index, nndex_cuda_ivf_stats* out) {
    clear_error();
    if (!index || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    const CudaIndex* ix = index->impl;
    *out = ix->ivf ? ix->ivf->stats : nndex_cuda_ivf_stats{};
    return NNDEX_OK;
}

int nndex_cuda_fp64_scores(nndex_cuda_index* index, const float* dev_queries_normalized, uint64_t query_rows,
                           const uint64_t* dev_pairs_query, const uint64_t* dev_pairs_row, uint64_t n,
                           double* dev_out) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    (void)query_rows;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    launch_fp64_pairs(ix->d_base, ix->ds, dev_queries_normalized, ix->dims, dev_pairs_query, dev_pairs_row, n, dev_out,
                      ix->stream);
    cudaError_t e = cudaStreamSynchronize(ix->stream);
    if (e != cudaSuccess) return cuda_error(e, "fp64 scores");
    return NNDEX_OK;
}

}  // extern "C"
