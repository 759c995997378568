// diagnostics.cu — checks of the failure handling that need no GPU fault.
//
// The reference has no counterpart: its GPU path waits without a limit (src/gpu.rs:573, 756
// `poll(wait_indefinitely)`). Every device-side wait in this library is bounded: after its budget
// of clock cycles a kernel records a timeout status and returns, the host reports
// NNDEX_ERR_TIMEOUT, and the context stays usable. nndex_cuda_check_bounded_wait runs one such
// wait on an mbarrier that nothing ever completes, so a test can watch the budget run out.
// nndex_cuda_inject_alloc_failures makes the next scratch allocations fail on the host side (no
// cudaMalloc is attempted), so out-of-memory handling can be tested without exhausting a GPU.
// nndex_cuda_plan_tc_ranges and nndex_cuda_plan_fp32_scan return the grids the scans would launch
// (host arithmetic only), so the planning rules are tested without a GPU.
#include "common.cuh"
#include "index.h"
#include "internal.h"

using namespace nndex;

namespace {

__global__ void bounded_wait_probe_kernel(long long budget, uint32_t* status) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    // No thread ever arrives on `bar`: the wait can only end by running out of its budget.
    if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, budget)) record_status(status, kStatusTimeout);
}

}  // namespace

extern "C" {

int nndex_cuda_check_bounded_wait(nndex_cuda_index* index, uint64_t budget_cycles) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    if (budget_cycles == 0 || budget_cycles > static_cast<uint64_t>(kWaitBudgetCycles))
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: wait budget must be 1..%lld cycles",
                         kWaitBudgetCycles);
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    cudaSetDevice(ix->device);
    ix->order_after_previous(ix->stream);
    cudaMemsetAsync(ix->d_status, 0, sizeof(uint32_t), ix->stream);
    bounded_wait_probe_kernel<<<1, 32, 0, ix->stream>>>(static_cast<long long>(budget_cycles), ix->d_status);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "wait check launch");
    ix->h_flags[0] = ~0ull;  // no validation error involved
    ix->h_flags[1] = 0;
    cudaMemcpyAsync(&ix->h_flags[1], ix->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ix->stream);
    cudaMemsetAsync(ix->d_status, 0, sizeof(uint32_t), ix->stream);
    ix->mark_done(ix->stream);
    if ((e = cudaStreamSynchronize(ix->stream)) != cudaSuccess) return cuda_error(e, "wait check");
    return ix->check_device_words();
}

void nndex_cuda_inject_alloc_failures(uint32_t count) { inject_alloc_failures(count); }

int nndex_cuda_plan_tc_ranges(uint64_t rows, uint64_t groups, uint32_t sm_count, uint64_t* nranges,
                              uint64_t* range_rows) {
    clear_error();
    if (!nranges || !range_rows || rows == 0 || groups == 0 || sm_count == 0)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: plan needs rows, groups and SMs");
    tc_range_split(rows, groups, sm_count, *nranges, *range_rows);
    return NNDEX_OK;
}

int nndex_cuda_plan_fp32_scan(uint32_t nq, uint32_t dims, uint32_t k, uint64_t rows, uint32_t sm_count,
                              uint64_t smem_limit, uint32_t* qb, uint32_t* groups, uint32_t* ctas_per_group) {
    clear_error();
    if (!qb || !groups || !ctas_per_group || dims == 0 || sm_count == 0)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: plan needs dims and SMs");
    ScanPlan plan;
    const uint32_t ds = (dims + 31) / 32 * 32;  // the stored row stride
    if (!plan_scan_fp32(nq, ds, k, rows, static_cast<int>(sm_count), static_cast<size_t>(smem_limit), plan))
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: no FP32 scan plan for nq=%u k=%u", nq, k);
    *qb = plan.qb;
    *groups = plan.groups;
    *ctas_per_group = plan.ctas_per_group;
    return NNDEX_OK;
}

}  // extern "C"
