// builder.cu — streaming construction and the .npy loader.
//
// The reference loads a matrix file into one Vec<f32> (src/python_io.rs:80-377) and hands it to
// NNdex::new, which copies it again while normalising (src/lib.rs:239-244). Here a matrix that
// arrives in pieces — a memory-mapped .npy, the arrays of an .npz, the record batches of a parquet
// column — streams through two pinned staging buffers straight into K1 (validate, normalise, pad,
// low-precision copies) on the device: no host copy of the whole matrix is ever made, and the
// upload of one piece overlaps the host's reading of the next.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>

#include "index.h"

using namespace nndex;

struct nndex_cuda_builder {
    CudaIndex* ix = nullptr;
    uint64_t rows = 0, dims = 0;
    uint64_t appended = 0;        // values received
    uint64_t chunk_rows = 0;      // rows per staging buffer
    float* h_stage[2] = {nullptr, nullptr};
    float* d_stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int b = 0;                    // staging buffer being filled
    uint64_t fill = 0;            // values in it
    uint64_t row0 = 0;            // first row it holds
    int failed = 0;               // first error, kept for finish

    ~nndex_cuda_builder() {
        if (ix) cudaSetDevice(ix->device);
        for (int i = 0; i < 2; ++i) {
            if (done[i]) {
                cudaEventSynchronize(done[i]);
                cudaEventDestroy(done[i]);
            }
            cudaFreeHost(h_stage[i]);
            cudaFree(d_stage[i]);
        }
        delete ix;
    }

    // Uploads the filled staging buffer (whole rows) and runs K1 on it; switches buffers.
    int flush() {
        if (fill == 0) return NNDEX_OK;
        const uint64_t n = fill / dims;
        cudaError_t e = cudaMemcpyAsync(d_stage[b], h_stage[b], fill * sizeof(float), cudaMemcpyHostToDevice,
                                        ix->stream);
        if (e != cudaSuccess) return cuda_error(e, "upload");
        index_prep_rows(ix, d_stage[b], row0, n);
        cudaEventRecord(done[b], ix->stream);
        row0 += n;
        fill = 0;
        b ^= 1;
        // the other buffer is reused only once its upload and K1 have finished
        if ((e = cudaEventSynchronize(done[b])) != cudaSuccess) return cuda_error(e, "upload");
        return NNDEX_OK;
    }
};

extern "C" {

int nndex_cuda_builder_begin(uint64_t rows, uint64_t dims, uint32_t flags, const nndex_cuda_opts* opts,
                             nndex_cuda_builder** out) {
    clear_error();
    if (!out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null output handle");
    *out = nullptr;
    if (rows == 0 || dims == 0) return err_shape(rows, dims, 0);
    auto* bld = new (std::nothrow) nndex_cuda_builder();
    if (!bld) return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: host allocation failed");
    int st = index_begin(rows, dims, flags, opts, &bld->ix);
    if (st) {
        delete bld;
        return st;
    }
    bld->rows = rows;
    bld->dims = dims;
    bld->chunk_rows = std::min<uint64_t>(rows, std::max<uint64_t>(1, (64ull << 20) / (dims * sizeof(float))));
    const size_t bytes = bld->chunk_rows * dims * sizeof(float);
    for (int i = 0; i < 2; ++i) {
        cudaError_t e;
        if ((e = cudaMallocHost(&bld->h_stage[i], bytes)) != cudaSuccess ||
            (e = cudaMalloc(&bld->d_stage[i], bytes)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&bld->done[i], cudaEventDisableTiming)) != cudaSuccess) {
            delete bld;
            return cuda_error(e, "staging buffers");
        }
    }
    *out = bld;
    return NNDEX_OK;
}

int nndex_cuda_builder_append(nndex_cuda_builder* bld, const float* host_values, uint64_t n_values) {
    clear_error();
    if (!bld) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null builder");
    if (bld->failed) return set_error(bld->failed, "%s", "cuda execution error: the build already failed");
    if (n_values == 0) return NNDEX_OK;
    if (!host_values) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null values");
    cudaSetDevice(bld->ix->device);
    if (bld->appended + n_values > bld->rows * bld->dims) {
        bld->failed = NNDEX_ERR_SHAPE_MISMATCH;
        return err_shape(bld->rows, bld->dims, bld->appended + n_values);
    }
    const uint64_t cap = bld->chunk_rows * bld->dims;
    uint64_t done = 0;
    while (done < n_values) {
        const uint64_t take = std::min(n_values - done, cap - bld->fill);
        std::memcpy(bld->h_stage[bld->b] + bld->fill, host_values + done, take * sizeof(float));
        bld->fill += take;
        done += take;
        if (bld->fill == cap) {
            const int st = bld->flush();
            if (st) {
                bld->failed = st;
                return st;
            }
        }
    }
    bld->appended += n_values;
    return NNDEX_OK;
}

int nndex_cuda_builder_finish(nndex_cuda_builder* bld, nndex_cuda_index** out) {
    clear_error();
    if (!bld || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    *out = nullptr;
    cudaSetDevice(bld->ix->device);
    int st = NNDEX_OK;
    // src/lib.rs:191: the shape is checked before anything the rows contain
    if (bld->failed == NNDEX_ERR_SHAPE_MISMATCH || bld->appended != bld->rows * bld->dims)
        st = err_shape(bld->rows, bld->dims, bld->appended);
    else if (bld->failed)
        st = set_error(bld->failed, "%s", "cuda execution error: the build failed while uploading");
    else
        st = bld->flush();
    if (st == NNDEX_OK) {
        CudaIndex* ix = bld->ix;
        bld->ix = nullptr;  // index_finish owns it now (and deletes it on failure)
        for (int i = 0; i < 2; ++i) cudaEventSynchronize(bld->done[i]);
        st = index_finish(ix);
        if (st == NNDEX_OK) *out = new nndex_cuda_index{ix};
    }
    delete bld;
    return st;
}

void nndex_cuda_builder_abort(nndex_cuda_builder* bld) { delete bld; }

// .npy (format 1.x-3.x) of little-endian float32, C order, two dimensions: memory-mapped and
// streamed through the builder.
int nndex_cuda_create_from_npy(const char* path, uint32_t flags, const nndex_cuda_opts* opts,
                               nndex_cuda_index** out) {
    clear_error();
    if (!path || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    *out = nullptr;
    auto bad = [&](const char* why) {
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "failed to read .npy matrix from '%s': %s", path, why);
    };
    const int fd = open(path, O_RDONLY);
    if (fd < 0) {
        const int en = errno;
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "failed to read .npy matrix from '%s': %s (os error %d)", path,
                         std::strerror(en), en);
    }
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
        close(fd);
        return bad("cannot stat the file");
    }
    const size_t size = static_cast<size_t>(sb.st_size);
    void* map = size ? mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0) : MAP_FAILED;
    close(fd);
    if (map == MAP_FAILED) return bad("cannot map the file");
    const unsigned char* p = static_cast<const unsigned char*>(map);
    auto unmap = [&](int code) {
        munmap(map, size);
        return code;
    };
    if (size < 10 || std::memcmp(p, "\x93NUMPY", 6) != 0) return unmap(bad("not a .npy file"));
    const int major = p[6];
    size_t hlen = 0, hoff = 0;
    if (major == 1) {
        hlen = p[8] | (p[9] << 8);
        hoff = 10;
    } else if (major == 2 || major == 3) {
        if (size < 12) return unmap(bad("truncated header"));
        hlen = p[8] | (p[9] << 8) | (static_cast<size_t>(p[10]) << 16) | (static_cast<size_t>(p[11]) << 24);
        hoff = 12;
    } else {
        return unmap(bad("unsupported format version"));
    }
    if (hoff + hlen > size) return unmap(bad("truncated header"));
    const std::string h(reinterpret_cast<const char*>(p + hoff), hlen);
    auto field = [&](const char* name) -> std::string {
        const size_t k = h.find(name);
        if (k == std::string::npos) return "";
        const size_t c = h.find(':', k);
        if (c == std::string::npos) return "";
        size_t v = c + 1;
        while (v < h.size() && h[v] == ' ') ++v;
        size_t e = v;
        if (h[v] == '(') e = h.find(')', v) + 1;
        else if (h[v] == '\'') e = h.find('\'', v + 1) + 1;
        else while (e < h.size() && h[e] != ',' && h[e] != '}') ++e;
        return h.substr(v, e - v);
    };
    const std::string descr = field("'descr'"), fortran = field("'fortran_order'"), shape = field("'shape'");
    if (descr != "'<f4'" && descr != "'=f4'") return unmap(bad("the array is not little-endian float32"));
    if (fortran != "False") return unmap(bad("the array is not in C order"));
    unsigned long long r = 0, c = 0;
    char tail = 0;
    if (std::sscanf(shape.c_str(), "(%llu, %llu%c", &r, &c, &tail) != 3 || tail != ')')
        return unmap(bad("the array is not two-dimensional"));
    if (r == 0 || c == 0)
        return unmap(set_error(NNDEX_ERR_SHAPE_MISMATCH, "matrix loaded from '%s' is empty or has zero dimensions", path));
    const size_t data = hoff + hlen;
    if (data + static_cast<size_t>(r) * c * sizeof(float) > size) return unmap(bad("the data is truncated"));
    const float* values = reinterpret_cast<const float*>(p + data);
    nndex_cuda_builder* bld = nullptr;
    int st = nndex_cuda_builder_begin(r, c, flags, opts, &bld);
    if (st) return unmap(st);
    const uint64_t total = static_cast<uint64_t>(r) * c, step = bld->chunk_rows * c;
    for (uint64_t v0 = 0; v0 < total && st == NNDEX_OK; v0 += step)
        st = nndex_cuda_builder_append(bld, values + v0, std::min(step, total - v0));
    if (st) {
        nndex_cuda_builder_abort(bld);
        return unmap(st);
    }
    st = nndex_cuda_builder_finish(bld, out);
    return unmap(st);
}

}  // extern "C"
