// Matrix-Market ingest on the device and binary snapshots of a graph.
//
// gv_mtx_parse replaces the reference's host reader readFile
// (src/reader/marketReader.cu:3-121) and CSR::readGraph / initializeCSR
// (src/dynamicStructure/csr.cu:55-78): the header (first line not starting
// with '%') gives rows, cols and entries; every later line gives "src dst
// [value]", 1-based.  Here the text is copied to the device once; newlines
// are counted per 4 KB tile, the tile counts scanned and every line start
// written by its tile, then one thread per line parses its integers (and
// value) with no host loop over the data.  Lines that start with '%' or hold
// no digits are skipped, as the reference skips '%' lines.
//
// gv_snapshot_save / gv_snapshot_load write and read a graph as a checksummed
// CSR file (offsets, destinations, weights), the checkpoint and epoch
// snapshot of a store; loading builds the store with gv_bulk_build_csr.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "store.cuh"
#include "prims.cuh"
#include "launch.hpp"
#include "../../include/gv_ingest.h"

namespace gv {
namespace {

constexpr uint32_t MTX_TILE = 4096;     // bytes per tile
constexpr int MTX_THREADS = 256;        // 16 bytes per thread
constexpr uint32_t MTX_PER_THREAD = MTX_TILE / MTX_THREADS;

__global__ void __launch_bounds__(MTX_THREADS) k_mtx_count(const char *__restrict__ text, uint64_t begin, uint64_t end,
                                                           uint32_t *__restrict__ tile_cnt) {
    __shared__ uint32_t red[MTX_THREADS / 32];
    const uint64_t t0 = begin + (uint64_t)blockIdx.x * MTX_TILE + threadIdx.x * MTX_PER_THREAD;
    uint32_t c = 0;
    for (uint32_t j = 0; j < MTX_PER_THREAD; ++j)
        if (t0 + j < end && text[t0 + j] == '\n') ++c;
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < MTX_THREADS / 32; ++i) t += red[i];
        tile_cnt[blockIdx.x] = t;
    }
}

// Writes the position of every newline of the tile at nl[tile_off + rank].
__global__ void __launch_bounds__(MTX_THREADS) k_mtx_starts(const char *__restrict__ text, uint64_t begin, uint64_t end,
                                                            const unsigned long long *__restrict__ tile_off,
                                                            unsigned long long *__restrict__ nl) {
    __shared__ uint32_t wsum[MTX_THREADS / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t t0 = begin + (uint64_t)blockIdx.x * MTX_TILE + threadIdx.x * MTX_PER_THREAD;
    uint32_t c = 0;
    for (uint32_t j = 0; j < MTX_PER_THREAD; ++j)
        if (t0 + j < end && text[t0 + j] == '\n') ++c;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(GV_FULL_MASK, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t w = 0; w < warp; ++w) before += wsum[w];
    unsigned long long at = tile_off[blockIdx.x] + before + incl - c;
    for (uint32_t j = 0; j < MTX_PER_THREAD; ++j)
        if (t0 + j < end && text[t0 + j] == '\n') nl[at++] = t0 + j;
}

__device__ __forceinline__ bool mtx_space(char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; }

// Unsigned decimal at p (after blanks); returns false without digits.
__device__ __forceinline__ bool mtx_uint(const char *text, uint64_t &p, uint64_t e, unsigned long long &out) {
    while (p < e && mtx_space(text[p])) ++p;
    unsigned long long v = 0;
    uint64_t q = p;
    while (q < e && text[q] >= '0' && text[q] <= '9' && q - p < 20) v = v * 10 + (unsigned long long)(text[q++] - '0');
    if (q == p) return false;
    p = q;
    out = v;
    return true;
}

// Decimal real (sign, digits, fraction, exponent), accumulated in fp64.
__device__ __forceinline__ bool mtx_real(const char *text, uint64_t &p, uint64_t e, double &out) {
    while (p < e && mtx_space(text[p])) ++p;
    uint64_t q = p;
    double sign = 1.0;
    if (q < e && (text[q] == '-' || text[q] == '+')) sign = text[q++] == '-' ? -1.0 : 1.0;
    double v = 0.0;
    int digits = 0, frac = 0;
    while (q < e && text[q] >= '0' && text[q] <= '9') { v = v * 10.0 + (text[q++] - '0'); ++digits; }
    if (q < e && text[q] == '.') {
        ++q;
        while (q < e && text[q] >= '0' && text[q] <= '9') { v = v * 10.0 + (text[q++] - '0'); ++digits; ++frac; }
    }
    if (!digits) return false;
    int ex = 0;
    if (q < e && (text[q] == 'e' || text[q] == 'E')) {
        uint64_t r = q + 1;
        int es = 1;
        if (r < e && (text[r] == '-' || text[r] == '+')) es = text[r++] == '-' ? -1 : 1;
        int ev = 0, ed = 0;
        while (r < e && text[r] >= '0' && text[r] <= '9' && ed < 6) { ev = ev * 10 + (text[r++] - '0'); ++ed; }
        if (ed) { ex = es * ev; q = r; }
    }
    const int p10 = ex - frac;
    double scale = 1.0;
    for (int i = 0; i < (p10 < 0 ? -p10 : p10) && i < 400; ++i) scale *= 10.0;
    out = sign * (p10 < 0 ? v / scale : v * scale);
    p = q;
    return true;
}

// Line i spans [start, nl[i]) with start = data begin or nl[i-1] + 1.
// ok[i] = 1 when it holds an entry; bad ids raise err.
__global__ void k_mtx_parse(const char *__restrict__ text, uint64_t begin, uint64_t end,
                            const unsigned long long *__restrict__ nl, uint64_t nlines, uint64_t rows, uint64_t cols,
                            int with_value, uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                            float *__restrict__ val, uint32_t *__restrict__ ok, uint32_t *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nlines; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p = i == 0 ? begin : nl[i - 1] + 1;
        const uint64_t e = nl[i];
        ok[i] = 0;
        while (p < e && mtx_space(text[p])) ++p;
        if (p >= e || text[p] == '%') continue;  // blank or comment line
        unsigned long long a = 0, b = 0;
        if (!mtx_uint(text, p, e, a) || !mtx_uint(text, p, e, b)) {
            atomicOr(err, 1u);  // a data line without two ids
            continue;
        }
        if (a < 1 || b < 1 || a > rows || b > cols || a > 0xFFFFFFFFull || b > 0xFFFFFFFFull) {
            atomicOr(err, 2u);
            continue;
        }
        double v = 1.0;
        if (with_value && !mtx_real(text, p, e, v)) atomicOr(err, 4u);
        src[i] = (uint32_t)(a - 1);
        dst[i] = (uint32_t)(b - 1);
        if (val) val[i] = (float)v;
        ok[i] = 1;
    }
}

__global__ void k_mtx_compact(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                              const float *__restrict__ val, const uint32_t *__restrict__ ok,
                              const unsigned long long *__restrict__ pos, uint64_t nlines, uint64_t cap,
                              uint32_t *__restrict__ osrc, uint32_t *__restrict__ odst, float *__restrict__ oval) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nlines; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!ok[i] || pos[i] >= cap) continue;
        osrc[pos[i]] = src[i];
        odst[pos[i]] = dst[i];
        if (oval && val) oval[pos[i]] = val[i];
    }
}

__global__ void k_mtx_ones(float *__restrict__ v, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) v[i] = 1.0f;
}

// Header parse on the host: banner (field, symmetry), then the size line.
bool mtx_header(const char *t, uint64_t len, gv_mtx_info *info, uint64_t *data_begin) {
    std::memset(info, 0, sizeof(*info));
    uint64_t p = 0;
    bool have_banner = false;
    while (p < len) {
        uint64_t e = p;
        while (e < len && t[e] != '\n') ++e;
        std::string line(t + p, t + e);
        if (!line.empty() && line[0] == '%') {
            if (!have_banner && line.rfind("%%MatrixMarket", 0) == 0) {
                have_banner = true;
                info->pattern = line.find("pattern") != std::string::npos;
                info->symmetric = line.find("symmetric") != std::string::npos ||
                                  line.find("hermitian") != std::string::npos;
            }
        } else {
            unsigned long long r = 0, c = 0, z = 0;
            if (std::sscanf(line.c_str(), "%llu %llu %llu", &r, &c, &z) == 3) {
                info->rows = r;
                info->cols = c;
                info->entries = z;
                *data_begin = e < len ? e + 1 : len;
                return true;
            }
            bool blank = true;
            for (char ch : line) blank = blank && (ch == ' ' || ch == '\t' || ch == '\r');
            if (!blank) return false;
        }
        p = e + 1;
    }
    return false;
}

}  // namespace
}  // namespace gv

using namespace gv;

extern "C" gv_status gv_mtx_parse(const char *text, uint64_t len, int mem, gv_mtx_info *info, uint32_t *src,
                                  uint32_t *dst, float *values, uint64_t cap, uint64_t *count, void *stream) {
    if (!text || !info || !count) { set_error("null argument"); return GV_ERR_INVALID; }
    if (mem != GV_MEM_HOST && mem != GV_MEM_DEVICE) { set_error("bad mem flag"); return GV_ERR_INVALID; }
    cudaStream_t s = (cudaStream_t)stream;
    // header from the first bytes (host copy when the text is on the device)
    std::vector<char> head;
    const char *ht = text;
    uint64_t hlen = len;
    if (mem == GV_MEM_DEVICE) {
        hlen = std::min<uint64_t>(len, 1ull << 20);
        head.resize(hlen);
        cudaError_t e = cudaMemcpyAsync(head.data(), text, hlen, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e, "mtx header");
        ht = head.data();
    }
    uint64_t begin = 0;
    if (!mtx_header(ht, hlen, info, &begin)) { set_error("no Matrix-Market size line"); return GV_ERR_INVALID; }
    if (info->rows == 0 || info->rows > 0xFFFFFFF0ull) { set_error("row count out of range"); return GV_ERR_INVALID; }
    *count = 0;
    if (!src) return GV_OK;  // header only
    if (!dst) { set_error("null argument"); return GV_ERR_INVALID; }
    if (begin >= len) return GV_OK;
    // device copy of the text (pinned staging is the caller's choice; pageable works)
    const char *dtext = text;
    std::vector<void *> owned;
    auto dalloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        owned.push_back(p);
        return p;
    };
    auto release = [&]() {
        for (void *p : owned) cudaFree(p);
        owned.clear();
    };
    gv_status st = GV_OK;
    if (mem == GV_MEM_HOST) {
        char *t = (char *)dalloc(len);
        if (!t) { set_error("mtx text allocation failed"); return GV_ERR_NOMEM; }
        cudaError_t e = cudaMemcpyAsync(t, text, len, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) { release(); return cuda_status(e, "mtx text"); }
        dtext = t;
    }
    const uint64_t span = len - begin;
    const uint64_t ntiles = (span + MTX_TILE - 1) / MTX_TILE;
    uint32_t *tile_cnt = (uint32_t *)dalloc(ntiles * 4 + 16);
    unsigned long long *tile_off = (unsigned long long *)dalloc((ntiles + 1) * 8);
    void *tmp = dalloc(scan_scratch_bytes(ntiles + 1) + 256);
    uint32_t *err = (uint32_t *)dalloc(16);
    if (!tile_cnt || !tile_off || !tmp || !err) { release(); set_error("mtx scratch allocation failed"); return GV_ERR_NOMEM; }
    GV_LAUNCH(k_mtx_count, (unsigned)ntiles, MTX_THREADS, 0, s, dtext, begin, len, tile_cnt);
    scan_exclusive_u32_to_u64(tile_cnt, tile_off, ntiles, tile_off + ntiles, tmp, s);
    unsigned long long nnl = 0;
    char last = '\n';
    cudaError_t e = cudaMemcpyAsync(&nnl, tile_off + ntiles, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last, dtext + len - 1, 1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { release(); return cuda_status(e, "mtx lines"); }
    const uint64_t nlines = nnl + (last != '\n' ? 1 : 0);  // a last line without its newline
    unsigned long long *nl = (unsigned long long *)dalloc(nlines * 8 + 16);
    uint32_t *lsrc = (uint32_t *)dalloc(nlines * 4 + 16), *ldst = (uint32_t *)dalloc(nlines * 4 + 16);
    uint32_t *ok = (uint32_t *)dalloc(nlines * 4 + 16);
    unsigned long long *pos = (unsigned long long *)dalloc((nlines + 1) * 8);
    const bool want_val = values && !info->pattern;
    float *lval = want_val ? (float *)dalloc(nlines * 4 + 16) : nullptr;
    void *tmp2 = dalloc(scan_scratch_bytes(nlines + 1) + 256);
    if (!nl || !lsrc || !ldst || !ok || !pos || !tmp2 || (want_val && !lval)) {
        release();
        set_error("mtx line allocation failed");
        return GV_ERR_NOMEM;
    }
    GV_LAUNCH(k_mtx_starts, (unsigned)ntiles, MTX_THREADS, 0, s, dtext, begin, len, (const unsigned long long *)tile_off,
              nl);
    if (last != '\n') {
        const unsigned long long endpos = len;
        cudaMemcpyAsync(nl + nnl, &endpos, 8, cudaMemcpyHostToDevice, s);
    }
    cudaMemsetAsync(err, 0, 4, s);
    GV_LAUNCH(k_mtx_parse, grid_for(nlines, 256, 148 * 16), 256, 0, s, dtext, begin, len, (const unsigned long long *)nl,
              nlines, info->rows, info->cols, want_val ? 1 : 0, lsrc, ldst, lval, ok, err);
    scan_exclusive_u32_to_u64(ok, pos, nlines, pos + nlines, tmp2, s);
    unsigned long long nent = 0;
    uint32_t herr = 0;
    e = cudaMemcpyAsync(&nent, pos + nlines, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { release(); return cuda_status(e, "mtx parse"); }
    if (herr) {
        release();
        set_error(herr & 2u ? "mtx entry id out of range" : herr & 1u ? "mtx data line without two ids"
                                                                       : "mtx entry without a value");
        return GV_ERR_INVALID;
    }
    *count = nent;
    if (nent > cap) {
        release();
        set_error("mtx entries exceed the output capacity");
        return GV_ERR_CAPACITY;
    }
    // outputs: device arrays in place, host arrays through device staging
    uint32_t *osrc = src, *odst = dst;
    float *oval = want_val ? values : nullptr;
    if (mem == GV_MEM_HOST) {
        osrc = (uint32_t *)dalloc(nent * 4 + 16);
        odst = (uint32_t *)dalloc(nent * 4 + 16);
        if (want_val) oval = (float *)dalloc(nent * 4 + 16);
        if (!osrc || !odst || (want_val && !oval)) { release(); set_error("mtx output allocation failed"); return GV_ERR_NOMEM; }
    }
    GV_LAUNCH(k_mtx_compact, grid_for(nlines, 256, 148 * 16), 256, 0, s, (const uint32_t *)lsrc, (const uint32_t *)ldst,
              (const float *)lval, (const uint32_t *)ok, (const unsigned long long *)pos, nlines, cap, osrc, odst, oval);
    if (mem == GV_MEM_HOST) {
        e = cudaMemcpyAsync(src, osrc, nent * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, odst, nent * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && want_val) e = cudaMemcpyAsync(values, oval, nent * 4, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess && values && info->pattern) {  // pattern files: every value is 1
        if (mem == GV_MEM_HOST) {
            for (uint64_t i = 0; i < nent; ++i) values[i] = 1.0f;
        } else {
            GV_LAUNCH(k_mtx_ones, grid_for(nent, 256, 148 * 16), 256, 0, s, values, nent);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    release();
    return cuda_status(e, "mtx out");
}

// ------------------------------------------------------------- snapshots
namespace {

struct SnapHeader {
    char magic[8];        // "GVSNAP\0\1"
    uint32_t version;     // 1
    uint32_t flags;       // bit 0 directed, bit 1 weighted
    uint32_t n;
    uint32_t block_size;
    uint64_t m;           // stored entries
    uint64_t checksum;    // FNV-1a 64 of the payload
    uint64_t reserved[3];
};
static_assert(sizeof(SnapHeader) == 64, "snapshot header is 64 bytes");
const char kSnapMagic[8] = {'G', 'V', 'S', 'N', 'A', 'P', 0, 1};

uint64_t fnv1a(uint64_t h, const void *data, size_t bytes) {
    const unsigned char *p = (const unsigned char *)data;
    for (size_t i = 0; i < bytes; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

extern "C" gv_status gv_snapshot_save(gv_graph *g, const char *path) {
    if (!g || !path) { set_error("null argument"); return GV_ERR_INVALID; }
    uint32_t n = 0;
    uint64_t m = 0;
    gv_status st = gv_num_vertices(g, &n);
    if (st == GV_OK) st = gv_num_edges(g, &m);
    if (st != GV_OK) return st;
    const bool weighted = g->cfg.weighted != 0;
    std::vector<uint64_t> off((size_t)n + 1);
    std::vector<uint32_t> dst(std::max<uint64_t>(m, 1));
    std::vector<float> w(weighted ? std::max<uint64_t>(m, 1) : 0);
    st = gv_export_csr(g, off.data(), dst.data(), weighted ? w.data() : nullptr, m, GV_MEM_HOST, nullptr);
    if (st != GV_OK) return st;
    SnapHeader h{};
    std::memcpy(h.magic, kSnapMagic, 8);
    h.version = 1;
    h.flags = (g->cfg.directed ? 1u : 0u) | (weighted ? 2u : 0u);
    h.n = n;
    h.block_size = g->cfg.block_size;
    h.m = m;
    uint64_t c = 1469598103934665603ull;
    c = fnv1a(c, off.data(), off.size() * 8);
    c = fnv1a(c, dst.data(), m * 4);
    if (weighted) c = fnv1a(c, w.data(), m * 4);
    h.checksum = c;
    FILE *f = std::fopen(path, "wb");
    if (!f) { set_error(std::string("cannot open ") + path); return GV_ERR_INVALID; }
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    ok = ok && std::fwrite(off.data(), 8, off.size(), f) == off.size();
    ok = ok && (m == 0 || std::fwrite(dst.data(), 4, m, f) == m);
    ok = ok && (!weighted || m == 0 || std::fwrite(w.data(), 4, m, f) == m);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) { set_error(std::string("write failed: ") + path); return GV_ERR_INVALID; }
    return GV_OK;
}

extern "C" gv_status gv_snapshot_load(const char *path, const gv_config *base, gv_graph **out) {
    if (!path || !out) { set_error("null argument"); return GV_ERR_INVALID; }
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) { set_error(std::string("cannot open ") + path); return GV_ERR_INVALID; }
    SnapHeader h{};
    bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, kSnapMagic, 8) == 0 && h.version == 1 &&
              h.n > 0;
    std::vector<uint64_t> off;
    std::vector<uint32_t> dst;
    std::vector<float> w;
    const bool weighted = (h.flags & 2u) != 0;
    if (ok) {
        off.resize((size_t)h.n + 1);
        dst.resize(std::max<uint64_t>(h.m, 1));
        if (weighted) w.resize(std::max<uint64_t>(h.m, 1));
        ok = std::fread(off.data(), 8, off.size(), f) == off.size();
        ok = ok && (h.m == 0 || std::fread(dst.data(), 4, h.m, f) == h.m);
        ok = ok && (!weighted || h.m == 0 || std::fread(w.data(), 4, h.m, f) == h.m);
    }
    std::fclose(f);
    if (!ok) { set_error(std::string("not a readable snapshot: ") + path); return GV_ERR_INVALID; }
    uint64_t c = 1469598103934665603ull;
    c = fnv1a(c, off.data(), off.size() * 8);
    c = fnv1a(c, dst.data(), h.m * 4);
    if (weighted) c = fnv1a(c, w.data(), h.m * 4);
    if (c != h.checksum || off[h.n] != h.m) { set_error("snapshot checksum mismatch"); return GV_ERR_INVALID; }
    for (uint64_t i = 0; i < h.m; ++i)
        if (dst[i] >= h.n) { set_error("snapshot entry out of range"); return GV_ERR_INVALID; }
    gv_config cfg;
    if (base) cfg = *base;
    else gv_config_init(&cfg, h.n);
    cfg.num_vertices = h.n;
    cfg.directed = h.flags & 1u;
    cfg.weighted = weighted ? 1 : 0;
    if (!base) cfg.block_size = h.block_size;
    if (cfg.max_batch_pairs < h.m) cfg.max_batch_pairs = h.m;
    gv_graph *g = nullptr;
    gv_status st = gv_create(&cfg, &g);
    if (st != GV_OK) return st;
    st = gv_bulk_build_csr(g, off.data(), dst.data(), weighted ? w.data() : nullptr, GV_MEM_HOST, nullptr);
    if (st == GV_OK) st = gv_synchronize(g, nullptr);
    if (st != GV_OK) {
        gv_destroy(g);
        return st;
    }
    *out = g;
    return GV_OK;
}

extern "C" gv_status gv_graph_from_mtx(const char *path, const gv_config *base, gv_graph **out) {
    if (!path || !out) { set_error("null argument"); return GV_ERR_INVALID; }
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) { set_error(std::string("cannot open ") + path); return GV_ERR_INVALID; }
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> text(len > 0 ? (size_t)len : 1);
    const bool ok = len > 0 && std::fread(text.data(), 1, (size_t)len, f) == (size_t)len;
    std::fclose(f);
    if (!ok) { set_error(std::string("cannot read ") + path); return GV_ERR_INVALID; }
    gv_mtx_info info;
    uint64_t cnt = 0;
    gv_status st = gv_mtx_parse(text.data(), (uint64_t)len, GV_MEM_HOST, &info, nullptr, nullptr, nullptr, 0, &cnt, nullptr);
    if (st != GV_OK) return st;
    gv_config cfg;
    if (base) cfg = *base;
    else gv_config_init(&cfg, (uint32_t)info.rows);
    cfg.num_vertices = (uint32_t)info.rows;
    const uint64_t cap = std::max<uint64_t>(info.entries, 1) + 16;
    std::vector<uint32_t> src(cap), dst(cap);
    std::vector<float> val(cfg.weighted ? cap : 0);
    st = gv_mtx_parse(text.data(), (uint64_t)len, GV_MEM_HOST, &info, src.data(), dst.data(),
                      cfg.weighted ? val.data() : nullptr, cap, &cnt, nullptr);
    if (st != GV_OK) return st;
    if (cfg.max_batch_pairs < cnt) cfg.max_batch_pairs = cnt;
    gv_graph *g = nullptr;
    st = gv_create(&cfg, &g);
    if (st != GV_OK) return st;
    // an undirected store keeps both directions, as the reader symmetrises
    // for !DIRECTED (marketReader.cu:55-62)
    st = gv_insert_edges(g, src.data(), dst.data(), cfg.weighted ? val.data() : nullptr, cnt, GV_MEM_HOST, nullptr);
    if (st == GV_OK) st = gv_synchronize(g, nullptr);
    if (st != GV_OK) {
        gv_destroy(g);
        return st;
    }
    *out = g;
    return GV_OK;
}
