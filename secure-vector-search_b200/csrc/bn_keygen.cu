// bn_keygen.cu -- key generation on the device: the H and S of a cluster
// drawn from its h_seed exactly as regenerate_h_s does on the host
// (crypto.rs:258-270): one ChaCha20Rng(h_seed) stream, first m * n1 draws
// of sample_fp for H (row-major), then S row by row, where every column j of
// a row takes one u32 draw and, when that draw is below the sparsity
// threshold, one more u32 for the sign (sample_sparse_pm1,
// crypto.rs:207-223).
//
// H is position-addressed: draw i is words 2i, 2i+1 of the stream (a draw
// equal to p would shift the rest; it is flagged, and the caller fails with
// BN_EDRAW, odds 2^-61 per draw).  S is not: whether a word is a column draw
// or a sign draw depends on every word before it.  The parse is a two-state
// machine (expecting a column draw / expecting a sign draw) whose behaviour
// over a run of words depends only on the state it starts in, so it is
// scanned in parallel:
//   1. every thread runs 16 keystream blocks through the machine from both
//      start states: (end state, column draws, selected draws) for each;
//      each CTA composes its 256 threads' maps in order into a tile map;
//   2. one CTA walks the tile maps from the stream's start state: each
//      tile's start state and the column-draw and entry counts before it;
//   3. every thread recomputes its blocks from its own start (the tile's
//      prefix composed with the maps of the threads before it) and writes
//      the entries it parses, in stream order, at their final positions,
//      and the row pointers of the rows that start in its words.
// Parsing stops after exactly m * n column draws; the word region scanned is
// sized for m * n / 4 entries (mean m * n * mu = m * n / 8), and a denser S
// is reported as an error rather than truncated.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "bn_kernels.cuh"

namespace bn {

namespace {

constexpr int KG_THREADS = 256;
constexpr uint32_t KG_BLOCKS = 16;  // keystream blocks one thread parses
constexpr uint64_t KG_TILE_BLOCKS = (uint64_t)KG_THREADS * KG_BLOCKS;

// H: thread per keystream block (8 draws).
__global__ void keygen_h_kernel(ChaChaKey key, uint64_t count, uint64_t* __restrict__ H, uint32_t* __restrict__ flags) {
    const uint64_t nblk = (count + 7) / 8;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t w[16];
        chacha20_block(key, b, w);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint64_t i = b * 8 + q;
            if (i < count) {
                uint64_t x = ((uint64_t)w[2 * q] | ((uint64_t)w[2 * q + 1] << 32)) & P;
                if (x == P) { atomicOr(flags, DRAW_HIT_P); x = 0; }
                H[i] = x;
            }
        }
    }
}

// The machine over a run of words, from both start states at once.
// st[s] / cols[s] / nnz[s]: state, column draws and selected draws so far
// for start state s (0 = a column draw is due, 1 = a sign draw is due).
__device__ __forceinline__ void parse16(const uint32_t w[16], uint32_t thr, uint32_t st[2], uint32_t cols[2],
                                        uint32_t nnz[2]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const bool sel = w[i] < thr;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (st[s] == 0) {
                cols[s] += 1;
                if (sel) { nnz[s] += 1; st[s] = 1; }
            } else {
                st[s] = 0;
            }
        }
    }
}

// Packed map of a thread's run: per start state, end state (bit 0), column
// draws (bits 1-12) and selected draws (bits 13-24); 16 blocks = 256 words.
__device__ __forceinline__ uint32_t pack_map(uint32_t st, uint32_t cols, uint32_t nnz) {
    return st | (cols << 1) | (nnz << 13);
}

struct KgMap {  // a composed map (counts grow past the packed width)
    uint32_t end[2];
    uint64_t cols[2], nnz[2];
};

__device__ __forceinline__ KgMap unpack_map(uint64_t v) {
    KgMap m;
    for (int s = 0; s < 2; ++s) {
        const uint32_t x = (uint32_t)(v >> (32 * s));
        m.end[s] = x & 1u;
        m.cols[s] = (x >> 1) & 0xfffu;
        m.nnz[s] = (x >> 13) & 0xfffu;
    }
    return m;
}

// f then g
__device__ __forceinline__ KgMap compose(const KgMap& f, const KgMap& g) {
    KgMap h;
    for (int s = 0; s < 2; ++s) {
        const uint32_t e = f.end[s];
        h.end[s] = g.end[e];
        h.cols[s] = f.cols[s] + g.cols[e];
        h.nnz[s] = f.nnz[s] + g.nnz[e];
    }
    return h;
}

// 1. thread maps and tile maps.  Thread t of the grid parses S blocks
// [t * 16, t * 16 + 16) (block indices relative to the first S block).
__global__ void __launch_bounds__(KG_THREADS)
keygen_s_maps_kernel(ChaChaKey key, uint64_t sblock0, uint64_t nblocks, uint32_t thr, uint64_t* __restrict__ tmap,
                     KgMap* __restrict__ tile) {
    const uint64_t t = (uint64_t)blockIdx.x * KG_THREADS + threadIdx.x;
    uint32_t st[2] = {0u, 1u}, cols[2] = {0u, 0u}, nnz[2] = {0u, 0u};
    for (uint32_t k = 0; k < KG_BLOCKS; ++k) {
        const uint64_t b = t * KG_BLOCKS + k;
        if (b >= nblocks) break;
        uint32_t w[16];
        chacha20_block(key, sblock0 + b, w);
        parse16(w, thr, st, cols, nnz);
    }
    const uint64_t packed = (uint64_t)pack_map(st[0], cols[0], nnz[0]) | ((uint64_t)pack_map(st[1], cols[1], nnz[1]) << 32);
    tmap[t] = packed;
    __shared__ uint64_t sm[KG_THREADS];
    sm[threadIdx.x] = packed;
    __syncthreads();
    if (threadIdx.x == 0) {  // compose the tile's maps in stream order
        KgMap acc = unpack_map(sm[0]);
        for (int i = 1; i < KG_THREADS; ++i) acc = compose(acc, unpack_map(sm[i]));
        tile[blockIdx.x] = acc;
    }
}

struct KgStart {
    uint32_t st;
    uint64_t cols, nnz;
};

// 2. the stream starts expecting a column draw; every tile's start, and
// whether the scanned words held the m * n column draws (*ok).
__global__ void keygen_s_tiles_kernel(const KgMap* __restrict__ tile, uint64_t ntiles, uint64_t need_cols,
                                      KgStart* __restrict__ start, uint32_t* __restrict__ ok) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t st = 0;
    uint64_t cols = 0, nnz = 0;
    for (uint64_t i = 0; i < ntiles; ++i) {
        start[i] = KgStart{st, cols, nnz};
        const KgMap& f = tile[i];
        cols += f.cols[st];
        nnz += f.nnz[st];
        st = f.end[st];
    }
    *ok = cols >= need_cols ? 1u : 0u;
}

// 3. entries and row pointers.  A selected column draw's sign is the next
// word, which for the last word of a thread's run lies in the next block.
__global__ void __launch_bounds__(KG_THREADS)
keygen_s_emit_kernel(ChaChaKey key, uint64_t sblock0, uint64_t nblocks, uint32_t thr, uint32_t n, uint64_t need_cols,
                     const uint64_t* __restrict__ tmap, const KgStart* __restrict__ start, uint64_t cap,
                     uint32_t* __restrict__ s_idx, int8_t* __restrict__ s_sign, uint64_t* __restrict__ rowptr,
                     uint32_t* __restrict__ overflow) {
    __shared__ KgStart tstart[KG_THREADS];
    const uint64_t t0 = (uint64_t)blockIdx.x * KG_THREADS;
    if (threadIdx.x == 0) {  // exclusive prefix of the tile's thread maps from the tile's start
        KgStart s = start[blockIdx.x];
        for (int i = 0; i < KG_THREADS; ++i) {
            tstart[i] = s;
            const KgMap f = unpack_map(tmap[t0 + i]);
            s.cols += f.cols[s.st];
            s.nnz += f.nnz[s.st];
            s.st = f.end[s.st];
        }
    }
    __syncthreads();
    const uint64_t t = t0 + threadIdx.x;
    KgStart s = tstart[threadIdx.x];
    if (s.cols >= need_cols) return;  // past the last row
    uint32_t st = s.st;               // 0: a column draw is due, 1: a sign draw is due
    bool pending = false;             // an entry of this run whose sign word is due
    uint64_t pending_pos = 0;
    uint32_t w[16];
    for (uint32_t k = 0; k <= KG_BLOCKS; ++k) {
        const uint64_t b = t * KG_BLOCKS + k;
        if (b >= nblocks) return;
        if (k == KG_BLOCKS) {  // the next run's first word: the sign of this run's last entry
            if (pending) {
                chacha20_block(key, sblock0 + b, w);
                if (pending_pos < cap) s_sign[pending_pos] = (w[0] & 1u) == 0 ? (int8_t)-1 : (int8_t)1;
            }
            return;
        }
        chacha20_block(key, sblock0 + b, w);
        for (int i = 0; i < 16; ++i) {
            if (st == 1) {  // a sign word: this run's entry, or (first word) the previous run's
                if (pending && pending_pos < cap) s_sign[pending_pos] = (w[i] & 1u) == 0 ? (int8_t)-1 : (int8_t)1;
                pending = false;
                st = 0;
                continue;
            }
            const uint64_t c = s.cols++;  // a column draw: row c / n, column c % n
            if (c >= need_cols) return;
            if (c % n == 0) rowptr[c / n] = s.nnz;
            if (w[i] < thr) {
                pending_pos = s.nnz++;
                if (pending_pos < cap) s_idx[pending_pos] = (uint32_t)(c % n);
                else atomicOr(overflow, 1u);
                pending = true;
                st = 1;
            }
            if (c + 1 == need_cols) rowptr[need_cols / n] = s.nnz;  // the total closes the row pointers
        }
    }
}

// Row pointers of one list placed in the concatenated CSR: dst[i] = base + src[i].
__global__ void rowptr_shift_kernel(const uint64_t* __restrict__ src, uint64_t count, uint64_t base,
                                    uint64_t* __restrict__ dst) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = base + src[i];
}

}  // namespace

void launch_rowptr_shift(const uint64_t* d_src, uint64_t count, uint64_t base, uint64_t* d_dst, cudaStream_t s) {
    if (!count) return;
    const unsigned grid = (unsigned)std::min<uint64_t>((count + 255) / 256, 148 * 8);
    rowptr_shift_kernel<<<grid, 256, 0, s>>>(d_src, count, base, d_dst);
}

void launch_keygen_h(const uint8_t seed[32], uint64_t count, uint64_t* d_H, uint32_t* d_flags, int num_sms,
                     cudaStream_t s) {
    if (!count) return;
    const uint64_t nblk = (count + 7) / 8;
    const unsigned grid = (unsigned)std::min<uint64_t>((nblk + 255) / 256, (uint64_t)num_sms * 16);
    keygen_h_kernel<<<grid, 256, 0, s>>>(chacha_key(seed), count, d_H, d_flags);
}

uint64_t keygen_s_blocks(uint64_t m, uint32_t n) {
    const uint64_t words = m * n + (m * n) / 4 + 16;  // column draws + sign draws of up to m n / 4 entries
    const uint64_t blocks = (words + 15) / 16;
    return (blocks + KG_TILE_BLOCKS - 1) / KG_TILE_BLOCKS * KG_TILE_BLOCKS;
}

uint64_t keygen_s_scratch_bytes(uint64_t m, uint32_t n) {
    const uint64_t blocks = keygen_s_blocks(m, n), tiles = blocks / KG_TILE_BLOCKS;
    return blocks / KG_BLOCKS * 8 + tiles * (sizeof(KgMap) + sizeof(KgStart)) + 256 * 3;
}

void launch_keygen_s(const uint8_t seed[32], uint64_t m, uint32_t n, uint32_t n1, uint32_t thr, void* d_scratch,
                     uint64_t cap, uint32_t* d_idx, int8_t* d_sign, uint64_t* d_rowptr, uint32_t* d_status,
                     cudaStream_t s) {
    if (!m) return;
    const ChaChaKey key = chacha_key(seed);
    const uint64_t sblock0 = m * n1 * 2 / 16;  // H takes 2 m n1 words (n1 is a multiple of 64)
    const uint64_t blocks = keygen_s_blocks(m, n), tiles = blocks / KG_TILE_BLOCKS;
    char* p = static_cast<char*>(d_scratch);
    uint64_t* tmap = reinterpret_cast<uint64_t*>(p);
    p += (blocks / KG_BLOCKS * 8 + 255) / 256 * 256;
    KgMap* tile = reinterpret_cast<KgMap*>(p);
    p += (tiles * sizeof(KgMap) + 255) / 256 * 256;
    KgStart* start = reinterpret_cast<KgStart*>(p);
    keygen_s_maps_kernel<<<(unsigned)tiles, KG_THREADS, 0, s>>>(key, sblock0, blocks, thr, tmap, tile);
    keygen_s_tiles_kernel<<<1, 32, 0, s>>>(tile, tiles, m * n, start, d_status);  // status[0]: the words held S
    keygen_s_emit_kernel<<<(unsigned)tiles, KG_THREADS, 0, s>>>(key, sblock0, blocks, thr, n, m * n, tmap, start, cap,
                                                                d_idx, d_sign, d_rowptr, d_status + 1);
}

}  // namespace bn
