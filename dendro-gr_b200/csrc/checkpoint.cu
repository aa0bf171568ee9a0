// Checkpoint and restart of an evolution: the reference's
// BSSNCtx::write_checkpt / restore_checkpt (BSSN_GR/src/bssnCtx.cpp:783-1170)
// for this library's mesh and zipped state.
//
//   <prefix>_step_<i>.cp         JSON header with the reference's keys (the
//                                reference writes it with nlohmann::json at
//                                indent 4: keys sorted, one per line)
//   <prefix>_octree_<i>_<r>.oct  "BSSNOCT1", nblocks, G[3], h, origin[3], the
//                                block descriptors, checksum
//   <prefix>_<i>_<r>.var         "BSSNVAR1", nvars, n_nodes, the variables
//                                (variable-major, n_nodes doubles each),
//                                checksum
//
// Every file is written to "<name>.tmp" and renamed when complete, so an
// interrupted write leaves the slot's previous checkpoint intact.  The
// variables move through a pinned host buffer in chunks, the device-to-host
// copy of one chunk overlapping the file write of the previous one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bssn_b200.h"

static_assert(sizeof(BssnBlockDesc) == 80, "block descriptor layout of the .oct file");

namespace {

constexpr char kOctMagic[8] = {'B', 'S', 'S', 'N', 'O', 'C', 'T', '1'};
constexpr char kVarMagic[8] = {'B', 'S', 'S', 'N', 'V', 'A', 'R', '1'};
constexpr size_t kChunkBytes = size_t(32) << 20;  // per pinned half-buffer

// Checksum over 8-byte words (the files are laid out in whole words):
// each word is xor-ed in and the state mixed by a multiply / xor-shift round.
struct Hash {
    uint64_t h = 0x6a09e667f3bcc908ull;
    void words(const void* p, size_t bytes) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        size_t n = bytes / 8;
        for (size_t i = 0; i < n; i++) {
            uint64_t w;
            std::memcpy(&w, c + 8 * i, 8);
            mix(w);
        }
        if (bytes % 8) {
            uint64_t w = 0;
            std::memcpy(&w, c + 8 * n, bytes % 8);
            mix(w ^ (uint64_t(bytes % 8) << 56));
        }
    }
    void mix(uint64_t w) {
        h ^= w;
        h *= 0x9fb21c651e98df25ull;
        h ^= h >> 29;
    }
};

std::string slot_name(const char* prefix, const char* mid, int index, int rank, const char* ext) {
    char buf[64];
    if (rank < 0)
        std::snprintf(buf, sizeof buf, "%s%d.%s", mid, index, ext);
    else
        std::snprintf(buf, sizeof buf, "%s%d_%d.%s", mid, index, rank, ext);
    return std::string(prefix) + buf;
}
std::string cp_name(const char* prefix, int index) { return slot_name(prefix, "_step_", index, -1, "cp"); }
std::string oct_name(const char* prefix, int index, int rank) {
    return slot_name(prefix, "_octree_", index, rank, "oct");
}
std::string var_name(const char* prefix, int index, int rank) {
    return slot_name(prefix, "_", index, rank, "var");
}

bool write_all(FILE* f, const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
bool read_all(FILE* f, void* p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }

// Finishes "<name>.tmp" -> name; removes the temporary on failure.
int commit_file(FILE* f, const std::string& name, bool ok) {
    const std::string tmp = name + ".tmp";
    ok = (std::fflush(f) == 0) && ok;
    ok = (std::fclose(f) == 0) && ok;
    if (ok && std::rename(tmp.c_str(), name.c_str()) != 0) ok = false;
    if (!ok) std::remove(tmp.c_str());
    return ok ? BSSN_OK : BSSN_EIO;
}

// Whether p is memory a CUDA copy must move (device or managed); host
// memory, or a process without a usable device, is copied directly.
bool device_pointer(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // clear the (non-sticky) error of the query
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Two pinned halves for the chunked copies (plain host memory when pinning
// is unavailable, which only happens without a device).
struct Staging {
    double* buf = nullptr;
    bool pinned = false;
    size_t half_doubles = kChunkBytes / sizeof(double);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int init(bool need_device) {
        if (need_device) {
            if (cudaHostAlloc(&buf, 2 * kChunkBytes, cudaHostAllocDefault) != cudaSuccess) return BSSN_ENOMEM;
            pinned = true;
            for (auto& e : ev)
                if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return BSSN_ENOMEM;
        } else {
            buf = static_cast<double*>(std::malloc(2 * kChunkBytes));
            if (!buf) return BSSN_ENOMEM;
        }
        return BSSN_OK;
    }
    ~Staging() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (pinned)
            cudaFreeHost(buf);
        else
            std::free(buf);
    }
    double* half(int k) { return buf + size_t(k) * half_doubles; }
};

// ---- JSON header (bssnCtx.cpp:829-857 writes these keys) ------------------
struct JsonKey {
    const char* name;
    int kind;  // 0 double, 1 int64, 2 int32
    size_t off;
};
#define JK(n, k, f) JsonKey{n, k, offsetof(BssnCheckpointInfo, f)}
// sorted as nlohmann::json prints an object
const JsonKey kKeys[] = {
    {"DENDRO_BH1_X", 0, offsetof(BssnCheckpointInfo, bh) + 0 * sizeof(double)},
    {"DENDRO_BH1_Y", 0, offsetof(BssnCheckpointInfo, bh) + 1 * sizeof(double)},
    {"DENDRO_BH1_Z", 0, offsetof(BssnCheckpointInfo, bh) + 2 * sizeof(double)},
    {"DENDRO_BH2_X", 0, offsetof(BssnCheckpointInfo, bh) + 3 * sizeof(double)},
    {"DENDRO_BH2_Y", 0, offsetof(BssnCheckpointInfo, bh) + 4 * sizeof(double)},
    {"DENDRO_BH2_Z", 0, offsetof(BssnCheckpointInfo, bh) + 5 * sizeof(double)},
    JK("DENDRO_TS_ACTIVE_COMM_SZ", 2, active_comm_size),
    JK("DENDRO_TS_ELEMENT_ORDER", 2, element_order),
    JK("DENDRO_TS_LAST_IO_TIME", 0, time_current),
    JK("DENDRO_TS_LOAD_IMB_TOLERANCE", 0, load_imb_tol),
    JK("DENDRO_TS_NUM_VARS", 2, num_vars),
    JK("DENDRO_TS_STEP_CURRENT", 1, step),
    JK("DENDRO_TS_TIME_BEGIN", 0, time_begin),
    JK("DENDRO_TS_TIME_CURRENT", 0, time_current),
    JK("DENDRO_TS_TIME_END", 0, time_end),
    JK("DENDRO_TS_TIME_STEP_SIZE", 0, time_step),
    JK("DENDRO_TS_WAVELET_TOLERANCE", 0, wavelet_tol),
};
#undef JK

int write_header(const char* prefix, int index, const BssnCheckpointInfo& info) {
    const std::string name = cp_name(prefix, index);
    FILE* f = std::fopen((name + ".tmp").c_str(), "w");
    if (!f) return BSSN_EIO;
    bool ok = std::fputs("{\n", f) >= 0;
    const int nk = int(sizeof(kKeys) / sizeof(kKeys[0]));
    for (int i = 0; i < nk && ok; i++) {
        const char* p = reinterpret_cast<const char*>(&info) + kKeys[i].off;
        const char* sep = i + 1 < nk ? "," : "";
        if (kKeys[i].kind == 0) {
            double v;
            std::memcpy(&v, p, sizeof v);
            ok = std::fprintf(f, "    \"%s\": %.17g%s\n", kKeys[i].name, v, sep) > 0;
        } else if (kKeys[i].kind == 1) {
            int64_t v;
            std::memcpy(&v, p, sizeof v);
            ok = std::fprintf(f, "    \"%s\": %lld%s\n", kKeys[i].name, (long long)v, sep) > 0;
        } else {
            int32_t v;
            std::memcpy(&v, p, sizeof v);
            ok = std::fprintf(f, "    \"%s\": %d%s\n", kKeys[i].name, (int)v, sep) > 0;
        }
    }
    ok = ok && std::fputs("}\n", f) >= 0;
    return commit_file(f, name, ok);
}

// Reads a header written by write_header (or any JSON object holding the
// keys as numbers).  BSSN_ENOENT when the file does not exist.
int read_header(const char* prefix, int index, BssnCheckpointInfo* info) {
    const std::string name = cp_name(prefix, index);
    FILE* f = std::fopen(name.c_str(), "r");
    if (!f) return errno == ENOENT ? BSSN_ENOENT : BSSN_EIO;
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    std::fclose(f);
    BssnCheckpointInfo out;
    std::memset(&out, 0, sizeof out);
    for (const JsonKey& k : kKeys) {
        const std::string quoted = std::string("\"") + k.name + "\"";
        const size_t at = text.find(quoted);
        if (at == std::string::npos) return BSSN_EIO;
        size_t c = at + quoted.size();
        while (c < text.size() && (text[c] == ' ' || text[c] == '\t' || text[c] == '\n' || text[c] == '\r')) c++;
        if (c >= text.size() || text[c] != ':') return BSSN_EIO;
        const char* s = text.c_str() + c + 1;
        char* end = nullptr;
        errno = 0;
        const double v = std::strtod(s, &end);
        if (end == s || errno == ERANGE || !std::isfinite(v)) return BSSN_EIO;
        char* p = reinterpret_cast<char*>(&out) + k.off;
        if (k.kind == 0) {
            std::memcpy(p, &v, sizeof v);
        } else {
            const long long iv = std::strtoll(s, &end, 10);
            if (k.kind == 1) {
                const int64_t w = iv;
                std::memcpy(p, &w, sizeof w);
            } else {
                const int32_t w = (int32_t)iv;
                std::memcpy(p, &w, sizeof w);
            }
        }
    }
    *info = out;
    return BSSN_OK;
}

}  // namespace

extern "C" {

int bssn_checkpoint_index(int64_t step, int freq, int merged, int* merged_written) {
    if (freq <= 0 || step < 0) return -1;
    if (merged && merged_written && !*merged_written) {
        *merged_written = 1;
        return 3;
    }
    return (step % (2 * int64_t(freq)) == 0) ? 0 : 1;
}

int bssn_checkpoint_write(const char* prefix, int index, int rank, int write_header_flag,
                          const BssnCheckpointInfo* info, const BssnBlockDesc* blocks,
                          int nblocks, const int32_t G[3], double h, const double origin[3],
                          const double* const* u_dev, int64_t n_nodes, bssn_stream_t stream) {
    if (!prefix || !info || (!blocks && nblocks) || nblocks < 0 || !G || !origin || !u_dev ||
        n_nodes < 0 || index < 0 || rank < 0)
        return BSSN_EINVAL;
    for (int v = 0; v < BSSN_NUM_VARS; v++)
        if (!u_dev[v] && n_nodes) return BSSN_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    // mesh
    {
        const std::string name = oct_name(prefix, index, rank);
        FILE* f = std::fopen((name + ".tmp").c_str(), "wb");
        if (!f) return BSSN_EIO;
        Hash hs;
        const int32_t head[4] = {nblocks, G[0], G[1], G[2]};
        const double geo[4] = {h, origin[0], origin[1], origin[2]};
        bool ok = write_all(f, kOctMagic, 8) && write_all(f, head, sizeof head) &&
                  write_all(f, geo, sizeof geo) &&
                  write_all(f, blocks, sizeof(BssnBlockDesc) * size_t(nblocks));
        hs.words(kOctMagic, 8);
        hs.words(head, sizeof head);
        hs.words(geo, sizeof geo);
        hs.words(blocks, sizeof(BssnBlockDesc) * size_t(nblocks));
        ok = ok && write_all(f, &hs.h, sizeof hs.h);
        const int st = commit_file(f, name, ok);
        if (st) return st;
    }
    // variables
    {
        bool dev = false;
        for (int v = 0; v < BSSN_NUM_VARS && n_nodes; v++) dev = dev || device_pointer(u_dev[v]);
        Staging stg;
        int st = stg.init(dev);
        if (st) return st;
        const std::string name = var_name(prefix, index, rank);
        FILE* f = std::fopen((name + ".tmp").c_str(), "wb");
        if (!f) return BSSN_EIO;
        const int32_t head[2] = {BSSN_NUM_VARS, 0};
        bool ok = write_all(f, kVarMagic, 8) && write_all(f, head, sizeof head) &&
                  write_all(f, &n_nodes, sizeof n_nodes);
        Hash hs;
        // chunk c of the concatenated variables goes through half c % 2; the
        // copy of chunk c + 1 is queued before chunk c is hashed and written
        std::vector<std::pair<int, int64_t>> chunks;  // (variable, first node)
        for (int v = 0; v < BSSN_NUM_VARS; v++)
            for (int64_t i = 0; i < n_nodes; i += int64_t(stg.half_doubles)) chunks.push_back({v, i});
        auto len = [&](size_t c) {
            return std::min<int64_t>(int64_t(stg.half_doubles), n_nodes - chunks[c].second);
        };
        auto fetch = [&](size_t c) -> bool {
            const double* src = u_dev[chunks[c].first] + chunks[c].second;
            double* dst = stg.half(int(c % 2));
            const size_t bytes = size_t(len(c)) * sizeof(double);
            if (!dev) {
                std::memcpy(dst, src, bytes);
                return true;
            }
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s) == cudaSuccess &&
                   cudaEventRecord(stg.ev[c % 2], s) == cudaSuccess;
        };
        if (!chunks.empty()) ok = ok && fetch(0);
        for (size_t c = 0; c < chunks.size() && ok; c++) {
            if (dev) ok = cudaEventSynchronize(stg.ev[c % 2]) == cudaSuccess;
            if (ok && c + 1 < chunks.size()) ok = fetch(c + 1);
            const size_t bytes = size_t(len(c)) * sizeof(double);
            hs.words(stg.half(int(c % 2)), bytes);
            ok = ok && write_all(f, stg.half(int(c % 2)), bytes);
        }
        ok = ok && write_all(f, &hs.h, sizeof hs.h);
        st = commit_file(f, name, ok);
        if (st) return st;
    }
    if (write_header_flag) return write_header(prefix, index, *info);
    return BSSN_OK;
}

int bssn_checkpoint_latest(const char* prefix, int* index, BssnCheckpointInfo* info) {
    if (!prefix || !index || !info) return BSSN_EINVAL;
    // restore_checkpt (bssnCtx.cpp:893-948): look at slots 0 and 1, take the
    // larger step, slot 0 on a tie
    BssnCheckpointInfo hi[2];
    int st[2];
    for (int i = 0; i < 2; i++) st[i] = read_header(prefix, i, &hi[i]);
    if (st[0] == BSSN_ENOENT && st[1] == BSSN_ENOENT) return BSSN_ENOENT;
    int pick;
    if (st[0] == BSSN_OK && st[1] == BSSN_OK)
        pick = hi[0].step < hi[1].step ? 1 : 0;
    else if (st[0] == BSSN_OK && st[1] == BSSN_ENOENT)
        pick = 0;
    else if (st[1] == BSSN_OK && st[0] == BSSN_ENOENT)
        pick = 1;
    else
        return BSSN_EIO;  // a header exists but does not parse
    *index = pick;
    *info = hi[pick];
    return BSSN_OK;
}

int bssn_checkpoint_read_mesh(const char* prefix, int index, int rank, BssnBlockDesc* blocks,
                              int* nblocks, int32_t G[3], double* h, double origin[3]) {
    if (!prefix || !nblocks || !G || !h || !origin || index < 0 || rank < 0) return BSSN_EINVAL;
    FILE* f = std::fopen(oct_name(prefix, index, rank).c_str(), "rb");
    if (!f) return errno == ENOENT ? BSSN_ENOENT : BSSN_EIO;
    char magic[8];
    int32_t head[4];
    double geo[4];
    bool ok = read_all(f, magic, 8) && std::memcmp(magic, kOctMagic, 8) == 0 &&
              read_all(f, head, sizeof head) && read_all(f, geo, sizeof geo) && head[0] >= 0;
    if (!ok) {
        std::fclose(f);
        return BSSN_EIO;
    }
    if (!blocks) {  // size query
        std::fclose(f);
        *nblocks = head[0];
        return BSSN_OK;
    }
    if (*nblocks < head[0]) {
        std::fclose(f);
        return BSSN_EINVAL;
    }
    std::vector<BssnBlockDesc> tmp(static_cast<size_t>(head[0]));
    uint64_t stored = 0;
    ok = read_all(f, tmp.data(), sizeof(BssnBlockDesc) * tmp.size()) && read_all(f, &stored, sizeof stored);
    std::fclose(f);
    if (!ok) return BSSN_EIO;
    Hash hs;
    hs.words(kOctMagic, 8);
    hs.words(head, sizeof head);
    hs.words(geo, sizeof geo);
    hs.words(tmp.data(), sizeof(BssnBlockDesc) * tmp.size());
    if (hs.h != stored) return BSSN_EIO;
    std::memcpy(blocks, tmp.data(), sizeof(BssnBlockDesc) * tmp.size());
    *nblocks = head[0];
    for (int d = 0; d < 3; d++) {
        G[d] = head[1 + d];
        origin[d] = geo[1 + d];
    }
    *h = geo[0];
    return BSSN_OK;
}

int bssn_checkpoint_read_vars(const char* prefix, int index, int rank, double* const* u_dev,
                              int64_t n_nodes, bssn_stream_t stream) {
    if (!prefix || !u_dev || n_nodes < 0 || index < 0 || rank < 0) return BSSN_EINVAL;
    for (int v = 0; v < BSSN_NUM_VARS; v++)
        if (!u_dev[v] && n_nodes) return BSSN_EINVAL;
    FILE* f = std::fopen(var_name(prefix, index, rank).c_str(), "rb");
    if (!f) return errno == ENOENT ? BSSN_ENOENT : BSSN_EIO;
    char magic[8];
    int32_t head[2];
    int64_t n = -1;
    bool ok = read_all(f, magic, 8) && std::memcmp(magic, kVarMagic, 8) == 0 &&
              read_all(f, head, sizeof head) && read_all(f, &n, sizeof n) && head[0] == BSSN_NUM_VARS;
    if (!ok) {
        std::fclose(f);
        return BSSN_EIO;
    }
    if (n != n_nodes) {
        std::fclose(f);
        return BSSN_EINVAL;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    bool dev = false;
    for (int v = 0; v < BSSN_NUM_VARS && n_nodes; v++) dev = dev || device_pointer(u_dev[v]);
    Staging stg;
    int st = stg.init(dev);
    if (st) {
        std::fclose(f);
        return st;
    }
    Hash hs;
    // chunk c is read into half c % 2 after the upload of chunk c - 2 from
    // that half has completed
    int64_t c = 0;
    for (int v = 0; v < BSSN_NUM_VARS && ok; v++) {
        for (int64_t i = 0; i < n_nodes && ok; i += int64_t(stg.half_doubles), c++) {
            const int64_t m = std::min<int64_t>(int64_t(stg.half_doubles), n_nodes - i);
            double* buf = stg.half(int(c % 2));
            if (dev && c >= 2) ok = cudaEventSynchronize(stg.ev[c % 2]) == cudaSuccess;
            ok = ok && read_all(f, buf, size_t(m) * sizeof(double));
            if (!ok) break;
            hs.words(buf, size_t(m) * sizeof(double));
            if (dev)
                ok = cudaMemcpyAsync(u_dev[v] + i, buf, size_t(m) * sizeof(double), cudaMemcpyDefault, s) ==
                         cudaSuccess &&
                     cudaEventRecord(stg.ev[c % 2], s) == cudaSuccess;
            else
                std::memcpy(u_dev[v] + i, buf, size_t(m) * sizeof(double));
        }
    }
    uint64_t stored = 0;
    ok = ok && read_all(f, &stored, sizeof stored);
    std::fclose(f);
    if (dev && cudaStreamSynchronize(s) != cudaSuccess) return BSSN_EIO;
    if (!ok || stored != hs.h) return BSSN_EIO;
    return BSSN_OK;
}

}  // extern "C"
