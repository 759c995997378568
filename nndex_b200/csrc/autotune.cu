// autotune.cu — the measured plan choice that replaces nndex's shape → strategy table
// (src/profiles.rs:65-185 TuningProfile::for_shape and cpu_batch_strategy, fixed thresholds on rows,
// dims and batch size).
//
// Every search path of this library returns the same bits for a query (fixed FMA orders, exact
// reranks behind certificates), so the choice between them is a pure speed question, and speed
// depends on the matrix, the batch and the device in ways fixed thresholds get wrong (the TF32
// candidate scan wins or loses against the FP32 scan depending on how clustered the data is; the
// tensor-core pass-1 stride trades pass-1 work against pass-2 collection). So the first batch of
// each shape runs every candidate plan twice (the first run pays one-time costs such as buffer
// growth), the second run is timed on the host clock around a synchronised stream, and the fastest
// plan is cached for the shape. A shape is (exact or IVF, queries rounded up to a power of two, k
// likewise, precision, nprobe); the matrix is the index's own.
//
// The cache can be exported as text and imported by a later process on the same device model for
// the same matrix shape and flags.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>

#include "index.h"

namespace nndex {

namespace {
uint32_t ceil_log2(uint64_t v) {
    uint32_t l = 0;
    while ((1ull << l) < v) ++l;
    return l;
}
constexpr const char* kHeader = "nndex-autotune v2";

// One shape of the key, as its fields.
struct ShapeFields {
    uint32_t ivf = 0, precision = 0, nprobe = 0;
    uint64_t nq = 0, k = 0;  // bucket values (powers of two)
};

uint64_t pack_key(const ShapeFields& f) {
    return static_cast<uint64_t>(f.ivf & 1u) | (static_cast<uint64_t>(ceil_log2(f.nq)) << 1) |
           (static_cast<uint64_t>(ceil_log2(f.k)) << 8) | (static_cast<uint64_t>(f.precision & 0xFFu) << 16) |
           (static_cast<uint64_t>(f.nprobe) << 24);
}

ShapeFields unpack_key(uint64_t key) {
    ShapeFields f;
    f.ivf = static_cast<uint32_t>(key & 1u);
    f.nq = 1ull << ((key >> 1) & 0x7Fu);
    f.k = 1ull << ((key >> 8) & 0xFFu);
    f.precision = static_cast<uint32_t>((key >> 16) & 0xFFu);
    f.nprobe = static_cast<uint32_t>(key >> 24);
    return f;
}

bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }

// Parses one entry line; false when malformed.
bool parse_entry(const char* line, uint64_t* key, CudaIndex::TuneEntry* e) {
    ShapeFields f;
    unsigned long long nq = 0, k = 0;
    int path = 0;
    unsigned stride = 0, qb = 0, ivf = 0, prec = 0, nprobe = 0;
    double ms = 0.0;
    int n = std::sscanf(line,
                        "shape ivf=%u nq=%llu k=%llu precision=%u nprobe=%u plan path=%d stride=%u qb=%u ms=%lf",
                        &ivf, &nq, &k, &prec, &nprobe, &path, &stride, &qb, &ms);
    if (n != 9 || ivf > 1 || !is_pow2(nq) || nq > kMaxBatchChunk || !is_pow2(k) || k > (1ull << 20) || prec > 3 ||
        path < 1 || path > 6 || stride > 64 || qb > 3 || !(ms >= 0.0))
        return false;
    if (ivf ? (path != 4 && path != 5) : (path == 4 || path == 5)) return false;
    if (path == 4 && stride) return false;
    if (qb && path != 2 && path != 3) return false;  // only the exact tensor-core pass 2 has two blocks
    f.ivf = ivf;
    f.nq = nq;
    f.k = k;
    f.precision = prec;
    f.nprobe = nprobe;
    *key = pack_key(f);
    e->plan.path = path;
    e->plan.stride = stride;
    e->plan.qb = qb;
    e->ms = ms;
    return true;
}

// Walks `text` line by line: the header first, then entries. Calls fn(key, entry) per entry.
template <class Fn>
int parse_cache(const char* text, std::string* header, Fn fn) {
    if (!text) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null autotune text");
    const char* p = text;
    uint64_t line_no = 0;
    bool have_header = false;
    while (*p) {
        const char* e = std::strchr(p, '\n');
        std::string line = e ? std::string(p, e - p) : std::string(p);
        p = e ? e + 1 : p + line.size();
        ++line_no;
        if (line.empty()) continue;
        if (!have_header) {
            if (line.compare(0, std::strlen(kHeader), kHeader) != 0)
                return set_error(NNDEX_ERR_INVALID_ARGUMENT,
                                 "cuda execution error: autotune text line %llu: expected the '%s' header",
                                 (unsigned long long)line_no, kHeader);
            if (header) *header = line;
            have_header = true;
            continue;
        }
        uint64_t key = 0;
        CudaIndex::TuneEntry ent;
        if (!parse_entry(line.c_str(), &key, &ent))
            return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: autotune text line %llu: bad entry '%s'",
                             (unsigned long long)line_no, line.c_str());
        fn(key, ent);
    }
    if (!have_header)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: autotune text has no header");
    return NNDEX_OK;
}

// The header an index writes and accepts: device model, matrix shape and construction flags.
std::string header_for(const CudaIndex& ix) {
    cudaDeviceProp prop;
    std::string name = "unknown";
    if (cudaGetDeviceProperties(&prop, ix.device) == cudaSuccess) name = prop.name;
    for (char& c : name)
        if (c == ' ') c = '_';
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s device=%s rows=%llu dims=%llu flags=%u", kHeader, name.c_str(),
                  (unsigned long long)ix.rows, (unsigned long long)ix.dims, ix.flags);
    return buf;
}
}  // namespace

uint64_t CudaIndex::tune_key(uint64_t nq, uint64_t kcap) const {
    ShapeFields f;
    f.ivf = uses_ivf() ? 1u : 0u;
    f.nq = 1ull << ceil_log2(std::max<uint64_t>(nq, 1));
    f.k = 1ull << ceil_log2(std::max<uint64_t>(kcap, 1));
    f.precision = precision;
    if (f.ivf)
        f.nprobe = static_cast<uint32_t>(ivf_scratch.nprobe ? ivf_scratch.nprobe
                                                            : ivf_choose_nprobe(ivf->nlist, kcap, rows));
    return pack_key(f);
}

CudaIndex::TunePlan CudaIndex::rule_plan(uint64_t nq, uint64_t kcap) const {
    TunePlan p;
    p.path = uses_ivf() ? ivf_path(nq, kcap) : choose_path(nq, kcap);
    return p;
}

std::vector<CudaIndex::TunePlan> CudaIndex::tune_candidates(uint64_t nq, uint64_t kcap) const {
    std::vector<TunePlan> c;
    auto tc_ok = [&](bool fp8) {
        if (fp8 ? !d_base_fp8 : !d_base_bf16) return false;
        const TcPlan p1 = plan_tc(kcap, fp8);
        return p1.kp >= kcap && p1.kp > 0 && plan_tc(0, fp8).stages > 0;
    };
    auto add_tc = [&](int path) {
        // pass 2 with one or two query blocks per CTA, where a batch has two blocks and they fit.
        // (CTA pairs, qb 3, are not timed: on 10M × 256 at 4,096 queries they tied one block in
        // BF16 and lost 17 % in FP8; an imported plan may still name them.)
        const bool pair = nq > 128 && tc_pair_stages_for(tc_chunks(path == 3), path == 3, smem_optin) > 0;
        for (uint32_t stride : {1u, 8u, 32u}) {
            if (stride > 1 && rows < 256ull * 64) break;  // sampled pass 1 (every 8th or 32nd tile) on large bases
            if (pair) {
                c.push_back({path, stride, 1});
                c.push_back({path, stride, 2});
            } else {
                c.push_back({path, stride, 0});
            }
        }
    };
    if (uses_ivf()) {
        c.push_back({4, 0});
        const TcPlan p1 = plan_tc(kcap, false);
        if (precision != NNDEX_PRECISION_FP32 && nq >= 64 && ivf->d_reordered16 && p1.kp >= kcap && p1.kp > 0 &&
            plan_tc(0, false).stages > 0) {
            // the tensor-core list scan with a full pass 1, or on every 2nd, 4th or 16th tile of its
            // lists (a denser sample gives a tighter T and fewer rows to re-score)
            c.push_back({5, 1});
            c.push_back({5, 2});
            c.push_back({5, 4});
            c.push_back({5, 16});
        }
        return c;
    }
    const bool tf32 = plan_tf32(nq, kcap).kp != 0;
    switch (precision) {
        case NNDEX_PRECISION_FP32:
            c.push_back({1, 0});
            if (tf32) c.push_back({6, 0});
            break;
        case NNDEX_PRECISION_BF16:
        case NNDEX_PRECISION_FP8: {
            const bool fp8 = precision == NNDEX_PRECISION_FP8;
            if (tc_ok(fp8)) add_tc(fp8 ? 3 : 2);
            else c.push_back({1, 0});
            break;
        }
        default:  // AUTO: the FP32 scans for small batches, the tensor cores beside them from 64
            if (nq <= 256) {
                c.push_back({1, 0});
                if (tf32) c.push_back({6, 0});
            }
            if (nq >= 64) {
                if (tc_ok(false)) add_tc(2);
                if (tc_ok(true)) add_tc(3);
            }
            if (c.empty()) c.push_back({1, 0});
            break;
    }
    return c;
}

CudaIndex::TunePlan CudaIndex::plan_for(uint64_t nq, uint64_t kcap, bool* measure) const {
    *measure = false;
    if (autotune) {
        auto it = tune_cache.find(tune_key(nq, kcap));
        if (it != tune_cache.end()) return it->second.plan;
        if (autotune == 1 && tune_candidates(nq, kcap).size() > 1) *measure = true;
    }
    return rule_plan(nq, kcap);
}

}  // namespace nndex

using namespace nndex;

extern "C" {

int nndex_cuda_set_autotune(nndex_cuda_index* index, int mode) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    if (mode < 0 || mode > 2) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: autotune mode %d", mode);
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    ix->autotune = mode;
    return NNDEX_OK;
}

int nndex_cuda_autotune_export(nndex_cuda_index* index, char* buf, uint64_t capacity, uint64_t* len) {
    clear_error();
    if (!index || !len) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    std::string out = header_for(*ix) + "\n";
    for (const auto& kv : ix->tune_cache) {
        const ShapeFields f = unpack_key(kv.first);
        char line[256];
        std::snprintf(line, sizeof(line),
                      "shape ivf=%u nq=%llu k=%llu precision=%u nprobe=%u plan path=%d stride=%u qb=%u ms=%.6f\n",
                      f.ivf, (unsigned long long)f.nq, (unsigned long long)f.k, f.precision, f.nprobe,
                      kv.second.plan.path, kv.second.plan.stride, kv.second.plan.qb, kv.second.ms);
        out += line;
    }
    *len = out.size() + 1;
    if (!buf) return NNDEX_OK;
    if (capacity < out.size() + 1)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: autotune buffer of %llu bytes, %zu needed",
                         (unsigned long long)capacity, out.size() + 1);
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return NNDEX_OK;
}

int nndex_cuda_autotune_import(nndex_cuda_index* index, const char* text) {
    clear_error();
    if (!index) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null index");
    CudaIndex* ix = index->impl;
    std::lock_guard<std::mutex> lock(ix->mu);
    std::string header;
    std::map<uint64_t, CudaIndex::TuneEntry> got;
    int st = parse_cache(text, &header, [&](uint64_t key, const CudaIndex::TuneEntry& e) { got[key] = e; });
    if (st) return st;
    const std::string mine = header_for(*ix);
    if (header != mine)
        return set_error(NNDEX_ERR_INVALID_ARGUMENT,
                         "cuda execution error: autotune text is for '%s', this index is '%s'", header.c_str(),
                         mine.c_str());
    for (const auto& kv : got) ix->tune_cache[kv.first] = kv.second;
    return NNDEX_OK;
}

int nndex_cuda_autotune_validate(const char* text, uint64_t* entries) {
    clear_error();
    uint64_t n = 0;
    const int st = parse_cache(text, nullptr, [&](uint64_t, const CudaIndex::TuneEntry&) { ++n; });
    if (entries) *entries = n;
    return st;
}

}  // extern "C"
