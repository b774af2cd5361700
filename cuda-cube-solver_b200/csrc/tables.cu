// libccs: building (BFS) and loading solving tables.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "bfs_kernel.cuh"
#include "ccs_internal.h"
#include "dispatch.cuh"

using namespace ccs;

namespace {

constexpr size_t CHUNK_BYTES = 256ull << 20;  // host staging for file I/O (the reference's 2^26 words)

struct PinnedBuffer {
    void* p = nullptr;
    explicit PinnedBuffer(size_t n) {
        if (cudaMallocHost(&p, n) != cudaSuccess) p = nullptr;
    }
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
};

void log_msg(ccs_log_fn log, const char* fmt, ...) {
    if (!log) return;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    log(buf);
}

// Two pinned staging buffers: the copy of one chunk overlaps the file I/O of the other.
struct Staging {
    PinnedBuffer a{CHUNK_BYTES}, b{CHUNK_BYTES};
    cudaEvent_t done[2] = {nullptr, nullptr};
    bool ok() const { return a.p && b.p && done[0] && done[1]; }
    Staging() {
        if (cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) != cudaSuccess) done[0] = nullptr;
        if (cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) != cudaSuccess) done[1] = nullptr;
    }
    ~Staging() {
        if (done[0]) cudaEventDestroy(done[0]);
        if (done[1]) cudaEventDestroy(done[1]);
    }
    void* buf(int i) const { return i ? b.p : a.p; }
};

int write_device_file(const void* dptr, uint64_t n_bytes, const std::string& path, cudaStream_t stream) {
    Staging st;
    if (!st.ok()) return fail(CCS_E_NOMEM, "pinned staging buffers");
    std::string tmp = path + ".tmp";  // a crash mid-write must not leave a table that looks complete
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail(CCS_E_FILE, "%s: cannot open for writing", tmp.c_str());
    const uint64_t n_chunks = (n_bytes + CHUNK_BYTES - 1) / CHUNK_BYTES;
    auto issue = [&](uint64_t c) -> cudaError_t {  // device -> staging buffer c % 2
        const uint64_t off = c * CHUNK_BYTES;
        const size_t n = (size_t)std::min<uint64_t>(CHUNK_BYTES, n_bytes - off);
        cudaError_t e = cudaMemcpyAsync(st.buf((int)(c & 1)), (const char*)dptr + off, n, cudaMemcpyDeviceToHost, stream);
        return e == cudaSuccess ? cudaEventRecord(st.done[c & 1], stream) : e;
    };
    cudaError_t e = n_chunks ? issue(0) : cudaSuccess;
    for (uint64_t c = 0; c < n_chunks && e == cudaSuccess; ++c) {
        if (c + 1 < n_chunks) e = issue(c + 1);
        if (e == cudaSuccess) e = cudaEventSynchronize(st.done[c & 1]);
        if (e != cudaSuccess) break;
        const size_t n = (size_t)std::min<uint64_t>(CHUNK_BYTES, n_bytes - c * CHUNK_BYTES);
        if (fwrite(st.buf((int)(c & 1)), 1, n, f) != n) {
            cudaStreamSynchronize(stream);
            fclose(f);
            return fail(CCS_E_FILE, "%s: write failed", tmp.c_str());
        }
    }
    if (e != cudaSuccess) {
        cudaStreamSynchronize(stream);
        fclose(f);
        return fail(CCS_E_CUDA, "copy to host: %s", cudaGetErrorString(e));
    }
    if (fclose(f) != 0) return fail(CCS_E_FILE, "%s: close failed", tmp.c_str());
    if (std::rename(tmp.c_str(), path.c_str()) != 0) return fail(CCS_E_FILE, "rename %s -> %s failed", tmp.c_str(), path.c_str());
    return CCS_OK;
}

// Reads `n_bytes` of `f` into device memory `d`, the read of one chunk overlapping the copy of
// the previous one.
int read_file_to_device(FILE* f, void* d, uint64_t n_bytes, const char* path, cudaStream_t stream) {
    Staging st;
    if (!st.ok()) return fail(CCS_E_NOMEM, "pinned staging buffers");
    for (uint64_t off = 0, c = 0; off < n_bytes; off += CHUNK_BYTES, ++c) {
        const size_t n = (size_t)std::min<uint64_t>(CHUNK_BYTES, n_bytes - off);
        void* b = st.buf((int)(c & 1));
        cudaError_t e = c >= 2 ? cudaEventSynchronize(st.done[c & 1]) : cudaSuccess;  // buffer's last copy done
        if (e == cudaSuccess && fread(b, 1, n, f) != n) {
            cudaStreamSynchronize(stream);
            return fail(CCS_E_FILE, "%s: short read", path);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync((char*)d + off, b, n, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaEventRecord(st.done[c & 1], stream);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(stream);
            return fail(CCS_E_CUDA, "copy to device: %s", cudaGetErrorString(e));
        }
    }
    CCS_CUDA_TRY(cudaStreamSynchronize(stream));
    return CCS_OK;
}

}  // namespace

extern "C" int ccs_load_table(ccs_handle* h, const char* kind, int format, const char* path) {
    if (!h || !kind || !path) return fail(CCS_E_ARG, "NULL argument");
    if (format != CCS_FMT_BLOCK && format != CCS_FMT_B3) return fail(CCS_E_ARG, "unknown table format %d", format);
    CCS_TRY(set_kind(h, kind));
    uint64_t want = table_bytes_for(h->kind, format);
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CCS_E_FILE, "%s not found", path);
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 0 || (uint64_t)size != want) {
        fclose(f);
        return fail(CCS_E_FILE, "%s: size %lld, expected %llu", path, size, (unsigned long long)want);
    }
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    free_table(h);
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, want) != cudaSuccess) {
        fclose(f);
        return fail(CCS_E_NOMEM, "device allocation of %llu bytes for the table", (unsigned long long)want);
    }
    const int rc = read_file_to_device(f, d, want, path, h->stream);
    if (rc != CCS_OK) {
        fclose(f);
        cudaFree(d);
        return rc;
    }
    fclose(f);
    h->d_table = d;
    h->table_bytes = want;
    h->format = format;
    return CCS_OK;
}

// The second resident table: same kind family as the first (class count, format), so one search
// kernel serves both; only the E-content class table (genc2) and the table pointer differ.
static int attach_second(ccs_handle* h, const char* kind, int format, uint32_t* d, uint64_t bytes) {
    KindDesc k2;
    CCS_TRY(get_kind(kind, &k2));
    if (!h->d_table || h->format != format || k2.mode != h->kind.mode || k2.nec != h->kind.nec)
        return fail(CCS_E_ARG, "a second table must match the first one's kind family and format");
    uint16_t genc[384];
    build_genc(k2, genc);
    CCS_CUDA_TRY(cudaMemcpy(reinterpret_cast<char*>(h->d_tables) + offsetof(DevTables, genc2), genc, sizeof genc,
                            cudaMemcpyHostToDevice));
    if (h->d_table2) cudaFree(h->d_table2);
    h->d_table2 = d;
    h->table2_bytes = bytes;
    h->kind2_name = kind;
    return CCS_OK;
}

extern "C" int ccs_attach_table(ccs_handle* h, const char* kind, int format, const char* path) {
    if (!h || !kind || !path) return fail(CCS_E_ARG, "NULL argument");
    if (!h->d_table) return fail(CCS_E_STATE, "load or build the first table before attaching a second one");
    KindDesc k2;
    CCS_TRY(get_kind(kind, &k2));
    uint64_t want = table_bytes_for(k2, format);
    const std::string path_s(path);
    FILE* f = fopen(path_s.c_str(), "rb");
    if (!f) return fail(CCS_E_FILE, "%s not found", path_s.c_str());
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 0 || (uint64_t)size != want) {
        fclose(f);
        return fail(CCS_E_FILE, "%s: size %lld, expected %llu", path_s.c_str(), size, (unsigned long long)want);
    }
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, want) != cudaSuccess) {
        fclose(f);
        return fail(CCS_E_NOMEM, "device allocation of %llu bytes for the second table", (unsigned long long)want);
    }
    int rc = read_file_to_device(f, d, want, path_s.c_str(), h->stream);
    fclose(f);
    if (rc != CCS_OK) {
        cudaFree(d);
        return rc;
    }
    rc = attach_second(h, kind, format, d, want);
    if (rc != CCS_OK) cudaFree(d);
    return rc;
}

extern "C" int ccs_last_build_passes(ccs_handle* h, ccs_bfs_pass* out, int max_out, int* n_out) {
    if (!h || !n_out || (max_out > 0 && !out)) return fail(CCS_E_ARG, "NULL argument");
    int n = (int)h->last_passes.size();
    for (int i = 0; i < n && i < max_out; ++i) out[i] = h->last_passes[i];
    *n_out = n;
    return CCS_OK;
}

// One BFS of `kind`, then the files of paths[CCS_FMT_BLOCK / _B3 / _MOD3] (NULL: not written) and,
// with keep_resident, the table of keep_format kept on the device (1: as the table, 2: as the
// second table).
// Puts a handle back on its resident table's kind when a build that did not replace that table
// leaves (on success and on every error path alike).
struct KindRestore {
    ccs_handle* h;
    std::string kind;
    bool active = true;
    ~KindRestore() {
        if (active && h->d_table && !kind.empty() && h->kind_name != kind) set_kind(h, kind.c_str());
    }
};

static int build_impl(ccs_handle* h, const char* kind, const char* const paths[3], int keep_format, int keep_resident,
                      uint64_t* depth_counts, int max_depths, int* n_depths, double* seconds, ccs_log_fn log) {
    const std::string first_kind = h->kind_ready ? h->kind_name : std::string();  // restored when a table stays
    KindRestore restore{h, first_kind};
    CCS_TRY(set_kind(h, kind));
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    const KindDesc k = h->kind;
    const uint64_t n_entries = k.n_entries;
    const uint64_t n_chunks = (n_entries + 15) / 16;
    auto t0 = std::chrono::steady_clock::now();

    // keep_resident 1: the new table replaces the handle's tables; 2: it becomes the second table.
    if (keep_resident == 2 && !h->d_table) return fail(CCS_E_STATE, "no first table to attach a second one to");
    if (keep_resident == 1) free_table(h);
    DeviceBuffer<uint8_t> depth(n_chunks * 16);
    DeviceBuffer<unsigned long long> counter(40);
    if (!depth.ok() || !counter.ok())
        return fail(CCS_E_NOMEM, "device allocation for the BFS (%llu bytes)", (unsigned long long)(n_chunks * 16));
    CCS_CUDA_TRY(cudaMemsetAsync(depth.p, 0xFF, n_chunks * 16, h->stream));
    CCS_CUDA_TRY(cudaMemsetAsync(counter.p, 0, 40 * sizeof(unsigned long long), h->stream));

    BfsParams P;
    P.depth = depth.p;
    P.n_entries = n_entries;
    P.n_chunks = n_chunks;
    P.classidx = h->d_classidx;
    P.class_rep = h->d_class_rep;
    P.class_stab = h->d_class_stab;
    P.counter = counter.p;
    const int grid = h->sms * 8;

    std::vector<uint64_t> counts;
    auto read_counter = [&](uint64_t* v) -> int {
        CCS_CUDA_TRY(cudaMemcpyAsync(v, counter.p, 8, cudaMemcpyDeviceToHost, h->stream));
        CCS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        CCS_CUDA_TRY(cudaMemsetAsync(counter.p, 0, 8, h->stream));
        return CCS_OK;
    };
    // per pass: entries found, random depth-byte reads, claim attempts, device time
    h->last_passes.clear();
    cudaEvent_t pe0, pe1;
    CCS_CUDA_TRY(cudaEventCreate(&pe0));
    CCS_CUDA_TRY(cudaEventCreate(&pe1));
    struct EventPair {
        cudaEvent_t a, b;
        ~EventPair() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } ev_guard{pe0, pe1};
    auto read_pass = [&](uint32_t d, bool fwd, uint64_t* found) -> int {
        unsigned long long c[3];
        CCS_CUDA_TRY(cudaMemcpyAsync(c, counter.p, sizeof c, cudaMemcpyDeviceToHost, h->stream));
        CCS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        CCS_CUDA_TRY(cudaMemsetAsync(counter.p, 0, sizeof c, h->stream));
        float ms = 0;
        CCS_CUDA_TRY(cudaEventElapsedTime(&ms, pe0, pe1));
        ccs_bfs_pass rec{};
        rec.depth = (int32_t)d + 1;
        rec.forward = fwd ? 1 : 0;
        rec.found = c[0];
        rec.random_reads = c[1];
        rec.claims = c[2];
        rec.seconds = ms * 1e-3;
        h->last_passes.push_back(rec);
        *found = c[0];
        return CCS_OK;
    };
    CCS_TRY(dispatch_kind(k, [&](auto M, auto N) {
        constexpr int MODE = decltype(M)::value, NEC = decltype(N)::value;
        bfs_seed<MODE, NEC><<<1, 32, 0, h->stream>>>(h->d_tables, P);
        CCS_CUDA_TRY(cudaGetLastError());
        uint64_t found = 0;
        CCS_TRY(read_counter(&found));
        counts.push_back(found);
        uint64_t remaining = n_entries - found;
        for (uint32_t d = 0; remaining; ++d) {
            if (d >= 30) return fail(CCS_E_CHECK, "BFS deeper than 30");
            // The reference's rule (table.py:112): forward while the frontier is under a
            // quarter of the unvisited entries, backward afterwards.
            bool forward = counts.back() < remaining / 4;
            auto ts = std::chrono::steady_clock::now();
            CCS_CUDA_TRY(cudaEventRecord(pe0, h->stream));
            if (forward) bfs_forward<MODE, NEC><<<grid, 256, 0, h->stream>>>(h->d_tables, P, d);
            else bfs_backward<MODE, NEC><<<grid, 256, 0, h->stream>>>(h->d_tables, P, d);
            CCS_CUDA_TRY(cudaGetLastError());
            CCS_CUDA_TRY(cudaEventRecord(pe1, h->stream));
            CCS_TRY(read_pass(d, forward, &found));
            double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
            log_msg(log, "depth %2u %s found %14llu (%7.2fs)", d + 1, forward ? "fwd" : "bwd", (unsigned long long)found, dt);
            if (found == 0) return fail(CCS_E_UNREACHABLE, "%llu entries unreachable", (unsigned long long)remaining);
            if (found > remaining) return fail(CCS_E_CHECK, "BFS found more entries than remain");
            counts.push_back(found);
            remaining -= found;
        }
        return CCS_OK;
    }));

    // Self-check: the histogram of depths equals the per-pass counts, nothing left unvisited.
    {
        DeviceBuffer<unsigned long long> hist(33);
        if (!hist.ok()) return fail(CCS_E_NOMEM, "histogram buffer");
        CCS_CUDA_TRY(cudaMemsetAsync(hist.p, 0, 33 * 8, h->stream));
        bfs_histogram<<<h->sms * 4, 256, 0, h->stream>>>(depth.p, n_entries, hist.p);
        CCS_CUDA_TRY(cudaGetLastError());
        unsigned long long hh[33];
        CCS_CUDA_TRY(cudaMemcpyAsync(hh, hist.p, sizeof hh, cudaMemcpyDeviceToHost, h->stream));
        CCS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < 33; ++i) {
            uint64_t want = i < (int)counts.size() ? counts[i] : 0;
            if (hh[i] != want)
                return fail(CCS_E_CHECK, "histogram of depth %d is %llu, BFS counted %llu", i, hh[i], (unsigned long long)want);
        }
    }

    // Encode: the block table always (the base-3 encoder reads its minima), the base-3 table when
    // it is written or kept, then the mod-3 file; each file through "<path>.tmp" and a rename.
    const uint64_t n_blk = (n_entries + BLOCK_ENTRIES - 1) / BLOCK_ENTRIES;
    const uint64_t n_b3 = (n_entries + B3_ENTRIES - 1) / B3_ENTRIES;
    DeviceBuffer<uint32_t> blk(n_blk * 8);
    if (!blk.ok()) return fail(CCS_E_NOMEM, "block table allocation");
    encode_block<<<h->sms * 8, 256, 0, h->stream>>>(depth.p, n_entries, n_blk, blk.p);
    CCS_CUDA_TRY(cudaGetLastError());
    const bool want_b3 = paths[CCS_FMT_B3] || (keep_resident && keep_format == CCS_FMT_B3);
    DeviceBuffer<uint32_t> b3(want_b3 ? n_b3 * 8 : 0);
    if (want_b3) {
        if (!b3.ok()) return fail(CCS_E_NOMEM, "base-3 table allocation");
        encode_b3<<<(unsigned)((n_b3 + 127) / 128), 128, 0, h->stream>>>(depth.p, blk.p, n_entries, n_b3, b3.p);
        CCS_CUDA_TRY(cudaGetLastError());
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(CCS_E_CUDA, "encoding the table: %s", cudaGetErrorString(e));
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (seconds) *seconds = secs;
    if (n_depths) *n_depths = (int)counts.size();
    if (depth_counts)
        for (int i = 0; i < (int)counts.size() && i < max_depths; ++i) depth_counts[i] = counts[i];

    if (paths[CCS_FMT_MOD3]) {
        DeviceBuffer<uint32_t> mod3(n_chunks);
        if (!mod3.ok()) return fail(CCS_E_NOMEM, "mod-3 table allocation");
        encode_mod3<<<h->sms * 8, 256, 0, h->stream>>>(depth.p, n_chunks, mod3.p);
        CCS_CUDA_TRY(cudaGetLastError());
        CCS_TRY(write_device_file(mod3.p, n_chunks * 4, paths[CCS_FMT_MOD3], h->stream));
    }
    if (paths[CCS_FMT_BLOCK]) CCS_TRY(write_device_file(blk.p, n_blk * 32, paths[CCS_FMT_BLOCK], h->stream));
    if (paths[CCS_FMT_B3]) CCS_TRY(write_device_file(b3.p, n_b3 * 32, paths[CCS_FMT_B3], h->stream));

    int rc = CCS_OK;
    if (keep_resident == 1 || keep_resident == 2) {
        DeviceBuffer<uint32_t>& kept = keep_format == CCS_FMT_B3 ? b3 : blk;
        const uint64_t kept_bytes = keep_format == CCS_FMT_B3 ? n_b3 * 32 : n_blk * 32;
        uint32_t* d_out = kept.release();
        if (keep_resident == 1) {
            free_table(h);
            h->d_table = d_out;
            h->table_bytes = kept_bytes;
            h->format = keep_format;
            restore.active = false;  // the new table is of the new kind
        } else {
            std::string second = h->kind_name;
            rc = set_kind(h, first_kind.c_str());  // the constants stay those of the first table's kind
            if (rc == CCS_OK) rc = attach_second(h, second.c_str(), keep_format, d_out, kept_bytes);
            if (rc != CCS_OK) cudaFree(d_out);
        }
    }
    return rc;
}

extern "C" int ccs_build_table(ccs_handle* h, const char* kind, int format, const char* out_path, int keep_resident,
                               uint64_t* depth_counts, int max_depths, int* n_depths, double* seconds,
                               ccs_log_fn log) {
    if (!h || !kind) return fail(CCS_E_ARG, "NULL argument");
    if (format != CCS_FMT_BLOCK && format != CCS_FMT_B3) return fail(CCS_E_ARG, "unknown table format %d", format);
    const char* paths[3] = {nullptr, nullptr, nullptr};
    paths[format] = out_path;
    return build_impl(h, kind, paths, format, keep_resident, depth_counts, max_depths, n_depths, seconds, log);
}

extern "C" int ccs_build_table_files(ccs_handle* h, const char* kind, const char* block_path, const char* b3_path,
                                     const char* mod3_path, uint64_t* depth_counts, int max_depths, int* n_depths,
                                     double* seconds, ccs_log_fn log) {
    if (!h || !kind) return fail(CCS_E_ARG, "NULL argument");
    if (!block_path && !b3_path && !mod3_path) return fail(CCS_E_ARG, "no file to write");
    const char* paths[3] = {block_path, b3_path, mod3_path};
    return build_impl(h, kind, paths, CCS_FMT_BLOCK, 0, depth_counts, max_depths, n_depths, seconds, log);
}

// Opens `path` and checks that it holds exactly `want` bytes.
static int open_sized(const char* path, uint64_t want, FILE** out) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CCS_E_FILE, "%s not found", path);
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 0 || (uint64_t)size != want) {
        fclose(f);
        return fail(CCS_E_FILE, "%s: size %lld, expected %llu", path, size, (unsigned long long)want);
    }
    *out = f;
    return CCS_OK;
}

static int read_sized(ccs_handle* h, const char* path, uint64_t n_bytes, DeviceBuffer<uint32_t>& d) {
    FILE* f = nullptr;
    CCS_TRY(open_sized(path, n_bytes, &f));
    const int rc = read_file_to_device(f, d.p, n_bytes, path, h->stream);
    fclose(f);
    return rc;
}

extern "C" int ccs_encode_b3_file(ccs_handle* h, const char* kind, const char* mod3_path, const char* block_path,
                                  const char* b3_path) {
    if (!h || !kind || !mod3_path || !block_path || !b3_path) return fail(CCS_E_ARG, "NULL argument");
    KindDesc k;
    CCS_TRY(get_kind(kind, &k));
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    const uint64_t n_entries = k.n_entries;
    const uint64_t n_words = (n_entries + 15) / 16;
    const uint64_t n_blk = (n_entries + BLOCK_ENTRIES - 1) / BLOCK_ENTRIES;
    const uint64_t n_b3 = (n_entries + B3_ENTRIES - 1) / B3_ENTRIES;
    DeviceBuffer<uint32_t> mod3(n_words), blk(n_blk * 8), b3(n_b3 * 8);
    if (!mod3.ok() || !blk.ok() || !b3.ok()) return fail(CCS_E_NOMEM, "device allocation for the base-3 encoding");
    CCS_TRY(read_sized(h, mod3_path, n_words * 4, mod3));
    CCS_TRY(read_sized(h, block_path, n_blk * 32, blk));
    encode_b3_mod3<<<(unsigned)((n_b3 + 127) / 128), 128, 0, h->stream>>>(mod3.p, blk.p, n_entries, n_b3, b3.p);
    CCS_CUDA_TRY(cudaGetLastError());
    CCS_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return write_device_file(b3.p, n_b3 * 32, b3_path, h->stream);
}

extern "C" int ccs_save_table(ccs_handle* h, int table, const char* path) {
    if (!h || !path) return fail(CCS_E_ARG, "NULL argument");
    if (table != 0 && table != 1) return fail(CCS_E_ARG, "table %d: 0 or 1", table);
    const uint32_t* d = table ? h->d_table2 : h->d_table;
    const uint64_t n = table ? h->table2_bytes : h->table_bytes;
    if (!d) return fail(CCS_E_STATE, "no table %d loaded", table);
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    return write_device_file(d, n, path, h->stream);
}

extern "C" int ccs_table_histogram(ccs_handle* h, int table, uint64_t* bins, int n_bins) {
    if (!h || !bins) return fail(CCS_E_ARG, "NULL argument");
    if (table != 0 && table != 1) return fail(CCS_E_ARG, "table %d: 0 or 1", table);
    if (n_bins < 1 || n_bins > 64) return fail(CCS_E_ARG, "n_bins %d: 1 to 64", n_bins);
    const uint32_t* d = table ? h->d_table2 : h->d_table;
    if (!d) return fail(CCS_E_STATE, "no table %d loaded", table);
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    DeviceBuffer<unsigned long long> out(64);
    if (!out.ok()) return fail(CCS_E_NOMEM, "histogram buffer");
    CCS_CUDA_TRY(cudaMemsetAsync(out.p, 0, 64 * 8, h->stream));
    // both tables share the kind's entry count (a second table matches the first's kind family)
    if (h->format == CCS_FMT_B3)
        table_histogram<FMT_B3><<<h->sms * 4, 256, 0, h->stream>>>(d, h->kind.n_entries, (uint32_t)n_bins, out.p);
    else
        table_histogram<FMT_BLOCK><<<h->sms * 4, 256, 0, h->stream>>>(d, h->kind.n_entries, (uint32_t)n_bins, out.p);
    CCS_CUDA_TRY(cudaGetLastError());
    unsigned long long hb[64];
    CCS_CUDA_TRY(cudaMemcpyAsync(hb, out.p, sizeof hb, cudaMemcpyDeviceToHost, h->stream));
    CCS_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n_bins; ++i) bins[i] = hb[i];
    return CCS_OK;
}
