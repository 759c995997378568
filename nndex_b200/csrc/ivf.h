// ivf.h — the IVF (inverted file) index of nndex's approximate mode, built and searched on the GPU.
//
// Reference: ApproxIndex (src/approx.rs:11-25) — centroids [nlist × dims], the matrix reordered so
// every cluster's rows are contiguous, original_indices (position → original row) and
// cluster_offsets [nlist + 1]. Built by k-means++ seeding (src/approx.rs:357-429) and spherical
// k-means (src/approx.rs:434-535); searched by probing the nprobe best clusters and reranking
// their rows exactly (src/approx.rs:159-215, src/cpu.rs:425-502).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/nndex_cuda.h"

namespace nndex {

struct CudaIndex;

// The built index: read-only once built, shared by every view of the CudaIndex (server slots).
struct IvfIndex {
    uint64_t nlist = 0;          // clusters (1 = single-list index, never probed)
    uint64_t iters = 0;          // k-means iterations
    uint64_t nlist_pad = 0;      // nlist rounded up to 256 (assignment GEMM tiles, dims-major stride)
    float* d_centroids = nullptr;  // nlist × ds FP32, final centroids (zero padded)
    float* d_cent_t = nullptr;     // ds × nlist_pad FP32, the same centroids dims-major (probe)
    float* d_reordered = nullptr;  // rows_alloc × ds FP32, cluster-contiguous copy of the base
    uint32_t* d_row_map = nullptr; // rows: reordered position → original row
    uint32_t* d_offsets = nullptr; // nlist + 1
    std::vector<uint64_t> h_offsets;
    std::vector<uint64_t> h_init_rows;  // rows chosen by k-means++ (diagnostics / parity)
    uint64_t max_list = 0;
    CUtensorMap tmap_reordered{};
    // BF16 copy of the reordered rows for the tensor-core list scan: kb16 = dims rounded up to 64,
    // per row an upper bound of ‖x − bf16(x)‖, and the largest of them.
    uint64_t kb16 = 0;
    __nv_bfloat16* d_reordered16 = nullptr;  // rows_alloc × kb16
    float* d_res16 = nullptr;                // rows (reordered order)
    float eps16 = 0.0f;
    CUtensorMap tmap_reordered16{};
    nndex_cuda_ivf_stats stats{};

    ~IvfIndex();
};

// Per-search scratch of the IVF path (one per CudaIndex view; grown on demand).
struct IvfScratch {
    uint32_t nprobe = 0;                // 0 = choose_nprobe per search
    uint32_t tc_stride = 1;             // tensor-core scan: pass 1 on every n-th tile (autotuned)
    uint32_t* d_probes = nullptr;       size_t cap_probes = 0;
    float* d_pscore = nullptr;          size_t cap_pscore = 0;     // B·nlist: centroid scores of the probe
    uint32_t* d_list_cnt = nullptr;     size_t cap_list_cnt = 0;   // nlist: queries probing each list
    uint32_t* d_list_fill = nullptr;    size_t cap_list_fill = 0;
    uint32_t* d_list_qoff = nullptr;    size_t cap_list_qoff = 0;  // nlist + 1
    uint32_t* d_item_off = nullptr;     size_t cap_item_off = 0;   // nlist + 1
    uint32_t* d_item_list = nullptr;    size_t cap_item_list = 0;  // tensor-core scan: list of each work item
    uint32_t* d_list_q = nullptr;       size_t cap_list_q = 0;     // B·nprobe: query of each (list, query) pair
    uint32_t* d_list_slot = nullptr;    size_t cap_list_slot = 0;  // B·nprobe: its first output slot
    uint32_t* d_q_slot_off = nullptr;   size_t cap_q_slot_off = 0; // B + 1
    unsigned long long* d_counters = nullptr; size_t cap_counters = 0;  // work counter, totals, rows probed
    uint64_t* d_ws = nullptr;           size_t cap_ws = 0;         // slots × k keys
    uint32_t* d_qblock_off = nullptr;   size_t cap_qblock_off = 0; // nlist + 1 (tensor-core scan)
    __nv_bfloat16* d_g16 = nullptr;     size_t cap_g16 = 0;        // gathered query blocks × 128 × kb16
    uint32_t* d_lane_qid = nullptr;     size_t cap_lane_qid = 0;   // gathered blocks × 128
    uint32_t* d_lane_slot = nullptr;    size_t cap_lane_slot = 0;
    unsigned long long* h_probed = nullptr;  // pinned [8]: FP32 scan: rows probed (Σ over queries), streamed, union

    ~IvfScratch();
};

// Builds the IVF of `ix` (k-means++ + spherical k-means + list layout) on the GPU. nlist, iters
// and the seed come from ix.opts (0 = the reference's policy). Returns an NNDEX status.
int ivf_build(CudaIndex& ix);

// Installs a saved IVF layout (the arrays nndex_cuda_ivf_layout exports: centroids nlist ×
// padded dims, offsets nlist + 1, original indices rows, k-means++ rows nlist or NULL) instead of
// building one; nlist 0 removes the IVF. Validates the arrays. Synchronises ix.stream.
int ivf_restore(CudaIndex& ix, uint64_t nlist, const float* centroids, const uint64_t* offsets,
                const uint64_t* original_indices, const uint64_t* init_rows);
// Position-sensitive 64-bit fingerprint of the stored (normalised, padded) rows.
int base_checksum(CudaIndex& ix, uint64_t* out);

// Enqueues the IVF search of `nq` normalised queries (stride ds) with capped k into the device
// outputs (rows of `k` slots), on the FP32 list scan. Returns an NNDEX status.
int ivf_search(CudaIndex& ix, const float* queries, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim,
               uint32_t* o_cnt, cudaStream_t s);
// The same result on the tensor cores: BF16 list scan with certified candidates, exact FP32 rerank
// (the queries of ix.d_qn and their BF16 copies ix.d_q_bf16 / ix.d_q_resid). Enqueues without a host
// round trip; ivf_finish_tc completes the batch once the stream has.
int ivf_search_tc(CudaIndex& ix, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                  cudaStream_t s);
// After the stream has completed an ivf_search_tc batch: statistics, the pass-1 stride rule, and an
// FP32 list-scan re-run of queries whose collection overflowed (patched into the outputs).
int ivf_finish_tc(CudaIndex& ix, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                  cudaStream_t s);

// src/approx.rs:305-311 choose_nlist and 318-336 choose_nprobe.
uint64_t ivf_choose_nlist(uint64_t rows);
uint64_t ivf_choose_nprobe(uint64_t nlist, uint64_t k, uint64_t rows);

}  // namespace nndex
