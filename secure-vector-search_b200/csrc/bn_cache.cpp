// bn_cache.cpp -- reader of the reference's on-disk BN-IVF cache
// (`.bntm-ivf-cache-<16 hex>.bin`), so that an index the reference built
// and encrypted can be loaded into this backend without re-running k-means
// or the encryption.
//
// File layout (scorer-bntm/src/ivf.rs:440-560 writes it, :1755-1901 reads
// it; offsets are absolute, integers little-endian):
//   header, 20 bytes (scorer-core/src/cache.rs:46-80):
//     magic "\x89SVScach" (8), version u32 = 1, fingerprint u64 =
//     FNV-1a 64 over the length-prefixed parameter parts
//   IVF payload (ivf-index/src/ivf.rs:68-89): dim u64, n_centroids u64,
//     centroids f32 [n_centroids][dim], n_clusters u64, then per cluster
//     size u64 and size x (id u32, vector f32 [dim])
//   zero padding to the next multiple of 8
//   n_clusters u64 (again), then per cluster: m u64, h_seed (32 bytes),
//     m_enc u64 [m][n], a_l u64 [m][n1], m_plain u64 [m][n], h u64 [m][n1]
//   l_subspace u64 [n][n1]
// S is not stored: the reference regenerates it from h_seed
// (crypto.rs:258-270), as callers of this reader do.
//
// The file is mapped read-only and indexed once; the copy functions gather
// the per-list regions into the concatenated list-order arrays that
// bn_ivf_build / bn_ivf_attach_client take.

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstring>
#include <vector>

#include "bn_b200.h"
#include "bn_host.h"

namespace bn {
namespace api {
int fail(int code, const char* fmt, ...);
}
}  // namespace bn

using bn::api::fail;

namespace {

constexpr uint8_t CACHE_MAGIC[8] = {0x89, 'S', 'V', 'S', 'c', 'a', 'c', 'h'};
constexpr uint32_t CACHE_VERSION = 1;

struct ListRegion {
    uint64_t m;
    uint64_t ids;      // first (id, vector) entry of the list in the payload
    uint64_t h_seed, m_enc, a_l, m_plain, h;
};

uint64_t rd64(const uint8_t* p) {
    uint64_t v;
    memcpy(&v, p, 8);
    return v;
}

}  // namespace

struct bn_ivf_cache {
    int fd = -1;
    const uint8_t* base = nullptr;
    uint64_t size = 0;
    uint32_t n = 0, n1 = 0;
    uint64_t dim = 0, nlist = 0, rows = 0, centroids = 0, l_subspace = 0;
    std::vector<ListRegion> lists;

    ~bn_ivf_cache() {
        if (base) munmap(const_cast<uint8_t*>(base), size);
        if (fd >= 0) close(fd);
    }
};

extern "C" {

uint64_t bn_host_cache_fingerprint(const uint8_t* const* parts, const uint64_t* lens, uint32_t nparts) {
    uint64_t h = 0xcbf29ce484222325ull;  // FNV-1a 64 offset basis
    auto eat = [&h](uint8_t b) {
        h ^= b;
        h *= 0x100000001b3ull;
    };
    for (uint32_t i = 0; i < nparts; ++i) {
        for (int k = 0; k < 8; ++k) eat((uint8_t)(lens[i] >> (8 * k)));  // length prefix, u64 LE
        for (uint64_t j = 0; j < lens[i]; ++j) eat(parts[i][j]);
    }
    return h;
}

int bn_host_ivf_cache_open(const char* path, uint64_t fingerprint, uint32_t n, uint32_t n1, bn_ivf_cache** out) {
    if (!path || !out) return fail(BN_EINVAL, "ivf cache: null argument");
    *out = nullptr;
    if (n == 0 || n1 == 0 || n1 > n) return fail(BN_EINVAL, "ivf cache: need 0 < n1 <= n");
    auto* c = new bn_ivf_cache();
    auto bad = [c](const char* why, unsigned long long at) {
        delete c;
        return fail(BN_EINVAL, "ivf cache: %s (byte %llu)", why, at);
    };
    c->fd = open(path, O_RDONLY);
    if (c->fd < 0) {
        delete c;
        return fail(BN_EINVAL, "ivf cache: cannot open %s", path);
    }
    struct stat st;
    if (fstat(c->fd, &st) != 0) return bad("cannot stat the file", 0);
    c->size = (uint64_t)st.st_size;
    if (c->size < 20) return bad("shorter than the 20-byte header", c->size);
    void* m = mmap(nullptr, c->size, PROT_READ, MAP_PRIVATE, c->fd, 0);
    if (m == MAP_FAILED) return bad("cannot map the file", 0);
    c->base = static_cast<const uint8_t*>(m);
    c->n = n;
    c->n1 = n1;
    const uint8_t* b = c->base;
    const uint64_t size = c->size;
    // every read below checks `need` bytes at `off` first
    auto have = [size](uint64_t off, uint64_t need) { return off <= size && need <= size - off; };

    if (memcmp(b, CACHE_MAGIC, 8) != 0) return bad("not a scorer cache file (magic)", 0);
    uint32_t version;
    memcpy(&version, b + 8, 4);
    if (version != CACHE_VERSION) return bad("unsupported cache version", 8);
    if (fingerprint && rd64(b + 12) != fingerprint) return bad("fingerprint differs from the expected parameters", 12);

    uint64_t off = 20;
    if (!have(off, 16)) return bad("truncated IVF payload header", off);
    c->dim = rd64(b + off);
    const uint64_t n_centroids = rd64(b + off + 8);
    off += 16;
    if (c->dim == 0 && n_centroids) return bad("centroids of dimension 0", off);
    if (c->dim > size / 4) return bad("vector dimension too large", off - 16);
    if (n_centroids > size / 4 || (c->dim && n_centroids > size / (4 * c->dim))) return bad("centroid count too large", off);
    c->centroids = off;
    if (!have(off, 4 * c->dim * n_centroids)) return bad("truncated centroids", off);
    off += 4 * c->dim * n_centroids;
    if (!have(off, 8)) return bad("truncated cluster count", off);
    c->nlist = rd64(b + off);
    off += 8;
    if (c->nlist != n_centroids) return bad("cluster count differs from the centroid count", off - 8);
    c->lists.resize(c->nlist);
    const uint64_t entry = 4 + 4 * c->dim;  // (id u32, vector f32 [dim])
    for (uint64_t l = 0; l < c->nlist; ++l) {
        if (!have(off, 8)) return bad("truncated cluster size", off);
        const uint64_t sz = rd64(b + off);
        off += 8;
        if (sz > size / entry || !have(off, sz * entry)) return bad("truncated cluster members", off);
        c->lists[l].m = sz;
        c->lists[l].ids = off;
        off += sz * entry;
        c->rows += sz;
    }
    off += (8 - off % 8) % 8;  // padding for the u64 regions
    if (!have(off, 8)) return bad("truncated BN cluster count", off);
    if (rd64(b + off) != c->nlist) return bad("BN cluster count differs from the IVF index", off);
    off += 8;
    for (uint64_t l = 0; l < c->nlist; ++l) {
        ListRegion& r = c->lists[l];
        if (!have(off, 40)) return bad("truncated list header", off);
        if (rd64(b + off) != r.m) return bad("list row count differs from the IVF membership", off);
        r.h_seed = off + 8;
        off += 40;
        const uint64_t wide = r.m * n * 8, narrow = r.m * n1 * 8;
        if (r.m > size / (8ull * n) || !have(off, 2 * wide + 2 * narrow)) return bad("truncated list arrays", off);
        r.m_enc = off;
        r.a_l = r.m_enc + wide;
        r.m_plain = r.a_l + narrow;
        r.h = r.m_plain + wide;
        off = r.h + narrow;
    }
    if (!have(off, 8ull * n * n1)) return bad("truncated l_subspace", off);
    c->l_subspace = off;
    *out = c;
    return BN_OK;
}

void bn_host_ivf_cache_close(bn_ivf_cache* c) { delete c; }

void bn_host_ivf_cache_info(const bn_ivf_cache* c, uint32_t* nlist, uint32_t* dim, uint64_t* rows) {
    if (nlist) *nlist = (uint32_t)c->nlist;
    if (dim) *dim = (uint32_t)c->dim;
    if (rows) *rows = c->rows;
}

void bn_host_ivf_cache_lists(const bn_ivf_cache* c, uint64_t* list_offsets, uint32_t* ids, float* centroids,
                             uint8_t* h_seeds) {
    uint64_t row = 0;
    const uint64_t entry = 4 + 4 * c->dim;
    if (centroids) memcpy(centroids, c->base + c->centroids, 4 * c->dim * c->nlist);
    for (uint64_t l = 0; l < c->nlist; ++l) {
        const ListRegion& r = c->lists[l];
        if (list_offsets) list_offsets[l] = row;
        if (ids)
            for (uint64_t i = 0; i < r.m; ++i) memcpy(ids + row + i, c->base + r.ids + i * entry, 4);
        if (h_seeds) memcpy(h_seeds + 32 * l, c->base + r.h_seed, 32);
        row += r.m;
    }
    if (list_offsets) list_offsets[c->nlist] = row;
}

void bn_host_ivf_cache_arrays(const bn_ivf_cache* c, uint64_t* m_enc, uint64_t* a_l, uint64_t* m_plain, uint64_t* h,
                              uint64_t* l_subspace) {
    uint64_t row = 0;
    const uint64_t n = c->n, n1 = c->n1;
    for (uint64_t l = 0; l < c->nlist; ++l) {
        const ListRegion& r = c->lists[l];
        if (m_enc) memcpy(m_enc + row * n, c->base + r.m_enc, r.m * n * 8);
        if (a_l) memcpy(a_l + row * n1, c->base + r.a_l, r.m * n1 * 8);
        if (m_plain) memcpy(m_plain + row * n, c->base + r.m_plain, r.m * n * 8);
        if (h) memcpy(h + row * n1, c->base + r.h, r.m * n1 * 8);
        row += r.m;
    }
    if (l_subspace) memcpy(l_subspace, c->base + c->l_subspace, n * n1 * 8);
}

}  // extern "C"
