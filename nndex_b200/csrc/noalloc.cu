// noalloc.cu — exact FP32 batch search for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc while they search: a serving process whose
// device memory is entirely reserved up front by another allocator (a framework's caching
// allocator or a fixed arena) has no free HBM for the library to grow its workspace into, and a
// latency-critical caller cannot take the implicit device-wide synchronisation that cudaMalloc and
// cudaFree may cause. nndex_cuda_search_batch_device_noalloc serves them: it runs the same kernels
// as nndex_cuda_search_batch_device, but every byte of scratch memory it needs (the normalised
// queries, the per-CTA candidate keys and the status words) lives in one file-scope device array
// of NNDEX_NOALLOC_SCRATCH_BYTES, which each GPU that loads this library holds until the process
// exits. The call allocates nothing: no cudaMalloc, cudaFree or allocating library routine.
//
// The array is shared by every call on a device and keeps the last call's contents; the status
// words that must start clean are reset by each call. Calls whose work overlaps on the GPU (from
// two threads, or on two streams) race on the array and must be serialised by the caller.
//
// Set-up: creating an index looks up the array's device address on the index's device, with that
// device current, through cudaGetSymbolAddress (host code cannot use the array's name as a device
// address) and caches it. With lazy module loading (the CUDA default since 12.2) that lookup is
// what loads the array onto the GPU, so its memory is taken when the index is created, alongside
// the index's own allocations, and never by a search. Batches run in pieces of at most 16,384
// queries (as the allocating entry point runs them), each reusing the array.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "index.h"
#include "internal.h"

namespace nndex {

static __device__ __align__(256) unsigned char g_noalloc_scratch[NNDEX_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (device < 0 || device >= kMaxDevices)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: device %d out of range", device);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
    return NNDEX_OK;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }
}  // namespace

int noalloc_bind(int device) {
    unsigned char* p = nullptr;
    return scratch_address(device, &p);
}

int search_device_noalloc(CudaIndex* ix, const float* d_queries, uint64_t nq, uint64_t k, uint64_t* d_idx_out,
                          float* d_sim_out, uint32_t* d_cnt_out, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaError_t e = cudaSetDevice(ix->device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    ix->stats = nndex_cuda_search_stats{};
    if (ix->uses_ivf())
        return set_error(NNDEX_ERR_UNSUPPORTED,
                         "cuda execution error: the no-allocation entry point serves exact indexes only");
    if (!s) s = cudaStreamLegacy;
    const uint64_t kcap = std::min<uint64_t>(k, ix->rows);
    // Batches run in pieces of at most kMaxBatchChunk queries, as the allocating entry point runs
    // them (the merge's grid holds one row of blocks per query); every piece reuses the array, so
    // the largest piece must fit.
    const uint64_t chunk_max = std::min<uint64_t>(nq, kMaxBatchChunk);
    const uint64_t chunk_last = nq - (nq - 1) / kMaxBatchChunk * kMaxBatchChunk;
    // Scratch layout: [status words | normalised queries | per-CTA candidate keys].
    const size_t words = 256;
    const size_t qbytes = align256(static_cast<size_t>(chunk_max) * ix->ds * sizeof(float));
    size_t wsbytes = 0;
    for (uint64_t n : {chunk_max, chunk_last}) {
        ScanPlan plan;
        if (kcap > kMaxFusedK ||
            !plan_scan_fp32(static_cast<uint32_t>(n), static_cast<uint32_t>(ix->ds), static_cast<uint32_t>(kcap),
                            ix->rows, ix->sm_count, ix->smem_optin, plan))
            return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: k=%llu above the fused top-k limit %u",
                             (unsigned long long)kcap, kMaxFusedK);
        wsbytes = std::max(wsbytes, static_cast<size_t>(plan.ctas_per_group) * kcap * n * sizeof(uint64_t));
    }
    const size_t need = words + qbytes + wsbytes;
    if (need > NNDEX_NOALLOC_SCRATCH_BYTES)
        return set_error(NNDEX_ERR_UNSUPPORTED,
                         "cuda execution error: %llu queries with k=%llu need %zu bytes of scratch, above the %zu "
                         "bytes the no-allocation entry point holds; split the batch",
                         (unsigned long long)chunk_max, (unsigned long long)kcap, need,
                         static_cast<size_t>(NNDEX_NOALLOC_SCRATCH_BYTES));
    unsigned char* scratch = nullptr;
    int st = scratch_address(ix->device, &scratch);
    if (st) return st;
    unsigned long long* d_err = reinterpret_cast<unsigned long long*>(scratch);
    uint32_t* d_status = reinterpret_cast<uint32_t*>(scratch + 8);
    float* d_qn = reinterpret_cast<float*>(scratch + words);
    uint64_t* d_ws = reinterpret_cast<uint64_t*>(scratch + words + qbytes);

    ix->order_after_previous(s);
    // From here on work is enqueued on the shared array: every return marks the stream, so the
    // next call (on any stream) is ordered after it.
    auto fail = [&](int code) {
        ix->mark_done(s);
        return code;
    };
    // The array keeps the previous call's contents: reset the words that must start clean.
    cudaMemsetAsync(d_err, 0xFF, sizeof(unsigned long long), s);
    cudaMemsetAsync(d_status, 0, sizeof(uint32_t), s);
    for (uint64_t q0 = 0; q0 < nq; q0 += kMaxBatchChunk) {
        const uint64_t n = std::min<uint64_t>(kMaxBatchChunk, nq - q0);
        ScanPlan pl;
        if (!plan_scan_fp32(static_cast<uint32_t>(n), static_cast<uint32_t>(ix->ds), static_cast<uint32_t>(kcap),
                            ix->rows, ix->sm_count, ix->smem_optin, pl))
            return fail(set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: no scan plan for %llu queries",
                                  (unsigned long long)n));
        const uint64_t per_query = static_cast<uint64_t>(pl.ctas_per_group) * kcap;
        PrepArgs p;
        p.src = d_queries + q0 * ix->dims;
        p.rows = n;
        p.dims = static_cast<uint32_t>(ix->dims);
        p.out = d_qn;
        p.out_stride = static_cast<uint32_t>(ix->ds);
        p.mode = ix->normalized ? 2 : 0;
        p.err = d_err;
        p.sm_count = ix->sm_count;
        launch_prep_rows(p, s);
        ScanArgs a;
        a.tmap = &ix->tmap_f32;
        a.tmap_tile = &ix->tmap_f32_176;
        a.tmap_112 = &ix->tmap_f32_112;
        a.queries = d_qn;
        a.nq = static_cast<uint32_t>(n);
        a.dq = static_cast<uint32_t>(ix->ds);
        a.rows = ix->rows;
        a.k = static_cast<uint32_t>(kcap);
        a.ws_keys = d_ws;
        a.status = d_status;
        if ((e = launch_scan_fp32(a, pl, s)) != cudaSuccess) return fail(cuda_error(e, "scan launch"));
        MergeArgs m;
        m.ws_keys = d_ws;
        m.nq = static_cast<uint32_t>(n);
        m.per_query = per_query;
        m.k = static_cast<uint32_t>(kcap);
        m.out_stride = static_cast<uint32_t>(kcap);
        m.idx_out = d_idx_out + q0 * kcap;
        m.sim_out = d_sim_out + q0 * kcap;
        m.count_out = d_cnt_out ? d_cnt_out + q0 : nullptr;
        if ((e = launch_merge_topk(m, s)) != cudaSuccess) return fail(cuda_error(e, "merge launch"));
        ix->stats.kernel_launches += 3;
        ix->stats.rows_scanned += ix->rows * n;
        ix->stats.scan_qb = pl.qb;
        ix->stats.scan_wide = pl.wide;
    }
    ix->stats.path = 1;
    // h_flags is pinned host memory the index allocated when it was created.
    ix->h_flags[1] = 0;
    cudaMemcpyAsync(&ix->h_flags[0], d_err, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&ix->h_flags[1], d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    ix->mark_done(s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "search");
    return ix->check_device_words();
}

}  // namespace nndex

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" int nndex_cuda_search_batch_device_noalloc(nndex_cuda_index* index, const float* dev_queries,
                                                      uint64_t query_rows, uint64_t query_dims, uint64_t k,
                                                      uint64_t* dev_idx_out, float* dev_sim_out,
                                                      uint32_t* dev_counts_out, void* stream) {
    using namespace nndex;
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    if (query_rows == 0 || query_dims != ix->dims) {
        return set_error(NNDEX_ERR_SHAPE_MISMATCH, "matrix shape mismatch: rows=%llu, dims=%llu, values=%llu",
                         (unsigned long long)query_rows, (unsigned long long)ix->dims,
                         (unsigned long long)(query_rows * query_dims));
    }
    if (k == 0) return set_error(NNDEX_ERR_INVALID_TOPK, "top-k must be greater than zero");
    if (!dev_queries || !dev_idx_out || !dev_sim_out)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null buffer");
    if (query_rows > 0xFFFFFFFFull)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: too many queries in one call");
    return search_device_noalloc(ix, dev_queries, query_rows, k, dev_idx_out, dev_sim_out, dev_counts_out,
                                 static_cast<cudaStream_t>(stream));
}
