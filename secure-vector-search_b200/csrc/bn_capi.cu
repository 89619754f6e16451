// bn_capi.cu -- implementation of the C ABI declared in include/bn_b200.h.
//
// Replaces the cudarc glue of the reference (scorer-bntm/src/gpu/mod.rs):
// instead of one synchronous H2D + launch + D2H per query and per probed
// list on the default stream (gpu/mod.rs:584-614), a query batch is packed
// into one pinned staging copy, the whole pipeline (scan, Protocol 2,
// decode, top-k) is enqueued on the handle's own stream, and one D2H brings
// back only the ranked hits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bn_b200.h"
#include "bn_host.h"
#include "bn_internal.cuh"
#include "bn_kernels.cuh"
#include "bn_tc.cuh"

using namespace bn;

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_err;
}  // namespace

int bn::api::fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

using namespace bn::api;

namespace bn {
namespace api {

int corpus_tmap(Corpus& c) {
    if (!c.rows) return BN_OK;
    cudaError_t e = make_tmap_u8(&c.tmap_m, c.m_enc.p, (uint64_t)N * 8, c.rows, TC_ROWS, TC_ROWS);
    if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map of m_enc: %s", cudaGetErrorString(e));
    return BN_OK;
}

int check_shape(uint32_t n, uint32_t n1) {
    if (n != N) return fail(BN_EINVAL, "dimension too large: n = %u, this backend is built for n = %u", n, N);
    if (!(n1 == 64 || n1 == 128 || n1 == 256 || n1 == 512))
        return fail(BN_EINVAL, "n1 = %u is not 1024 >> k for k in 1..=4 (params.rs:102-120)", n1);
    return BN_OK;
}

// Row-major host [rows][cols] -> device column-major [cols][rows].
int upload_colmajor(bn_ctx* ctx, const uint64_t* host, uint64_t rows, uint32_t cols, DevMem& dst, cudaStream_t s) {
    TRY(dst.alloc(ctx, rows * cols * 8));
    if (rows == 0) return BN_OK;
    uint64_t chunk = std::max<uint64_t>(32, (256ull << 20) / (cols * 8ull));
    chunk = std::min(chunk, rows);
    DevMem tmp;
    TRY(tmp.alloc(ctx, chunk * cols * 8));
    for (uint64_t r0 = 0; r0 < rows; r0 += chunk) {
        uint64_t cr = std::min(chunk, rows - r0);
        CU(cudaMemcpyAsync(tmp.p, host + r0 * cols, cr * cols * 8, cudaMemcpyHostToDevice, s));
        launch_transpose_u64(tmp.at<uint64_t>(), cr, cols, dst.at<uint64_t>() + r0, rows, s);
        CU(cudaStreamSynchronize(s));
    }
    CU(cudaGetLastError());
    return BN_OK;
}

// Device row-major -> device column-major (whole array).
int device_colmajor(bn_ctx* ctx, const uint64_t* d_src, uint64_t rows, uint32_t cols, DevMem& dst, cudaStream_t s) {
    TRY(dst.alloc(ctx, rows * cols * 8));
    if (rows) launch_transpose_u64(d_src, rows, cols, dst.at<uint64_t>(), rows, s);
    CU(cudaGetLastError());
    return BN_OK;
}

// Sliced ELL of S from its row pointers (host, for the slice widths) and
// its entries already on the device.
int ell_from_device_csr(bn_ctx* ctx, const uint64_t* h_rowptr, const uint64_t* d_rowptr, const uint32_t* d_idx,
                        const int8_t* d_sign, uint64_t rows, Corpus& c, cudaStream_t s) {
    const uint64_t slices = (rows + 31) / 32;
    std::vector<uint16_t> w(std::max<uint64_t>(slices, 1), 0);
    std::vector<uint32_t> off(std::max<uint64_t>(slices, 1), 0);
    uint64_t total = 0;
    for (uint64_t sl = 0; sl < slices; ++sl) {
        uint64_t mx = 0;
        for (uint64_t i = sl * 32; i < std::min(rows, sl * 32 + 32); ++i) mx = std::max<uint64_t>(mx, h_rowptr[i + 1] - h_rowptr[i]);
        if (mx > N) return fail(BN_EINVAL, "S row with %llu entries exceeds n", (unsigned long long)mx);
        w[sl] = (uint16_t)mx;
        off[sl] = (uint32_t)total;
        total += mx * 32;
        if (total > 0xffffffffull) return fail(BN_EINVAL, "S too large for the sliced-ELL layout");
    }
    TRY(c.s_ell.alloc(ctx, std::max<uint64_t>(total, 1) * 2));
    TRY(c.s_off.alloc(ctx, off.size() * 4));
    TRY(c.s_w.alloc(ctx, w.size() * 2));
    CU(cudaMemcpyAsync(c.s_off.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c.s_w.p, w.data(), w.size() * 2, cudaMemcpyHostToDevice, s));
    if (rows)
        launch_csr_to_ell(d_rowptr, d_idx, d_sign, rows, c.s_off.at<uint32_t>(), c.s_w.at<uint16_t>(),
                          c.s_ell.at<uint16_t>(), s);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

int upload_sparse_ell(bn_ctx* ctx, bn_sparse_csr S, uint64_t rows, Corpus& c, cudaStream_t s) {
    const uint64_t slices = (rows + 31) / 32;
    std::vector<uint16_t> w(std::max<uint64_t>(slices, 1), 0);
    std::vector<uint32_t> off(std::max<uint64_t>(slices, 1), 0);
    uint64_t total = 0;
    for (uint64_t sl = 0; sl < slices; ++sl) {
        uint64_t mx = 0;
        for (uint64_t i = sl * 32; i < std::min(rows, sl * 32 + 32); ++i) {
            if (S.rowptr[i + 1] < S.rowptr[i]) return fail(BN_EINVAL, "s_mat.rowptr is not monotone at row %llu", (unsigned long long)i);
            mx = std::max<uint64_t>(mx, S.rowptr[i + 1] - S.rowptr[i]);
        }
        if (mx > N) return fail(BN_EINVAL, "s_mat row with %llu entries exceeds n", (unsigned long long)mx);
        w[sl] = (uint16_t)mx;
        off[sl] = (uint32_t)total;
        total += mx * 32;
        if (total > 0xffffffffull) return fail(BN_EINVAL, "s_mat too large for the sliced-ELL layout");
    }
    const uint64_t nnz = rows ? S.rowptr[rows] : 0;
    for (uint64_t e = 0; e < nnz; ++e)
        if (S.idx[e] >= N || (S.sign[e] != 1 && S.sign[e] != -1))
            return fail(BN_EINVAL, "s_mat entry %llu is not (col < n, sign +-1)", (unsigned long long)e);
    TRY(c.s_ell.alloc(ctx, std::max<uint64_t>(total, 1) * 2));
    TRY(c.s_off.alloc(ctx, off.size() * 4));
    TRY(c.s_w.alloc(ctx, w.size() * 2));
    CU(cudaMemcpyAsync(c.s_off.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c.s_w.p, w.data(), w.size() * 2, cudaMemcpyHostToDevice, s));
    if (rows) {
        DevMem rp, ix, sg;
        TRY(rp.alloc(ctx, (rows + 1) * 8));
        TRY(ix.alloc(ctx, std::max<uint64_t>(nnz, 1) * 4));
        TRY(sg.alloc(ctx, std::max<uint64_t>(nnz, 1)));
        CU(cudaMemcpyAsync(rp.p, S.rowptr, (rows + 1) * 8, cudaMemcpyHostToDevice, s));
        if (nnz) {
            CU(cudaMemcpyAsync(ix.p, S.idx, nnz * 4, cudaMemcpyHostToDevice, s));
            CU(cudaMemcpyAsync(sg.p, S.sign, nnz, cudaMemcpyHostToDevice, s));
        }
        launch_csr_to_ell(rp.at<uint64_t>(), ix.at<uint32_t>(), sg.at<int8_t>(), rows, c.s_off.at<uint32_t>(),
                          c.s_w.at<uint16_t>(), c.s_ell.at<uint16_t>(), s);
        CU(cudaGetLastError());
        CU(cudaStreamSynchronize(s));
    }
    return BN_OK;
}

int validate_residues(const uint64_t* a, uint64_t count, const char* what) {
    for (uint64_t i = 0; i < count; ++i)
        if (a[i] >= P) return fail(BN_EINVAL, "%s[%llu] = %llu is not a canonical residue mod 2^61-1", what,
                                   (unsigned long long)i, (unsigned long long)a[i]);
    return BN_OK;
}

// The decode's 32-row-blocked copies of [AL | H] and (for int8-valued
// plaintext) M, built once the client state is on the device.
int build_decode_layout(bn_ctx* ctx, Corpus& c, cudaStream_t s) {
    const uint64_t rows32 = (c.rows + 31) / 32 * 32;
    TRY(c.alh_b.alloc(ctx, rows32 * 2 * c.n1 * 8));
    TRY(c.m8_cm.alloc(ctx, rows32 * N));
    DevMem bad;
    TRY(bad.alloc(ctx, 4));
    launch_decode_layout(c.al_cm.at<uint64_t>(), c.h_cm.at<uint64_t>(), c.mp_cm.at<uint64_t>(), c.rows, c.n1,
                         c.alh_b.at<uint64_t>(), c.m8_cm.at<int8_t>(), bad.at<uint32_t>(), s);
    CU(cudaGetLastError());
    uint32_t hb = 0;
    CU(cudaMemcpyAsync(&hb, bad.p, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (hb) c.m8_cm.release();  // M T from the residues
    return BN_OK;
}

DecodeCorpus decode_corpus(const Corpus& c) {
    return DecodeCorpus{c.alh_b.at<uint64_t>(), c.m8_cm.p ? c.m8_cm.at<int8_t>() : nullptr, c.mp_cm.at<uint64_t>(),
                        c.s_ell.at<uint16_t>(), c.s_off.at<uint32_t>(), c.s_w.at<uint16_t>(),
                        c.ids.p ? c.ids.at<uint32_t>() : nullptr, c.rows, c.n1};
}

int attach_client(bn_ctx* ctx, Corpus& c, const uint64_t* L, const uint64_t* m_plain, bn_sparse_csr S, cudaStream_t s) {
    if (!L || !m_plain || (c.rows && (!S.rowptr || (S.rowptr[c.rows] && (!S.idx || !S.sign)))))
        return fail(BN_EINVAL, "attach_client: l_subspace, m_plain and s_mat are required");
    TRY(validate_residues(L, (uint64_t)N * c.n1, "l_subspace"));
    TRY(c.L.alloc(ctx, (uint64_t)N * c.n1 * 8));
    CU(cudaMemcpyAsync(c.L.p, L, (uint64_t)N * c.n1 * 8, cudaMemcpyHostToDevice, s));
    TRY(upload_colmajor(ctx, m_plain, c.rows, N, c.mp_cm, s));
    TRY(upload_sparse_ell(ctx, S, c.rows, c, s));
    CU(cudaStreamSynchronize(s));
    TRY(build_decode_layout(ctx, c, s));
    c.client = true;
    return BN_OK;
}

// Device encryption: m_enc = m_q + H L^T + S (row-major, stays on device in
// `m_enc`), AL = m_q L (row-major in `al_rm`).  crypto.rs:405-478.
int device_encrypt_dev(bn_ctx* ctx, const uint64_t* d_mq, uint64_t rows, uint32_t n1, const uint64_t* d_L,
                       const uint64_t* d_H, const uint64_t* d_rowptr, const uint32_t* d_idx, const int8_t* d_sign,
                       DevMem& m_enc, DevMem& al_rm, cudaStream_t s) {
    TRY(m_enc.alloc(ctx, rows * N * 8));
    TRY(al_rm.alloc(ctx, rows * n1 * 8));
    if (!rows) return BN_OK;
    launch_gemm_abt(d_H, d_L, d_mq, rows, N, n1, m_enc.at<uint64_t>(), s);  // H L^T + M
    launch_apply_sparse(d_rowptr, d_idx, d_sign, rows, N, m_enc.at<uint64_t>(), s);  // + S
    DevMem lt;  // AL = M L: B operand is L^T (n1 x n), K = n
    TRY(lt.alloc(ctx, (uint64_t)n1 * N * 8));
    launch_transpose_u64(d_L, N, n1, lt.at<uint64_t>(), N, s);
    launch_gemm_abt(d_mq, lt.at<uint64_t>(), nullptr, rows, n1, N, al_rm.at<uint64_t>(), s);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

int device_encrypt(bn_ctx* ctx, const uint64_t* d_mq, uint64_t rows, uint32_t n1, const uint64_t* d_L,
                   const uint64_t* d_H, bn_sparse_csr S, DevMem& m_enc, DevMem& al_rm, cudaStream_t s) {
    TRY(m_enc.alloc(ctx, rows * N * 8));
    TRY(al_rm.alloc(ctx, rows * n1 * 8));
    if (!rows) return BN_OK;
    // H L^T + M, K = n1
    launch_gemm_abt(d_H, d_L, d_mq, rows, N, n1, m_enc.at<uint64_t>(), s);
    CU(cudaGetLastError());
    {
        const uint64_t nnz = S.rowptr[rows];
        DevMem rp, ix, sg;
        TRY(rp.alloc(ctx, (rows + 1) * 8));
        TRY(ix.alloc(ctx, std::max<uint64_t>(nnz, 1) * 4));
        TRY(sg.alloc(ctx, std::max<uint64_t>(nnz, 1)));
        CU(cudaMemcpyAsync(rp.p, S.rowptr, (rows + 1) * 8, cudaMemcpyHostToDevice, s));
        if (nnz) {
            CU(cudaMemcpyAsync(ix.p, S.idx, nnz * 4, cudaMemcpyHostToDevice, s));
            CU(cudaMemcpyAsync(sg.p, S.sign, nnz, cudaMemcpyHostToDevice, s));
        }
        launch_apply_sparse(rp.at<uint64_t>(), ix.at<uint32_t>(), sg.at<int8_t>(), rows, N, m_enc.at<uint64_t>(), s);
        CU(cudaGetLastError());
        CU(cudaStreamSynchronize(s));
    }
    // AL = M L: B operand is L^T (n1 x n), K = n
    DevMem lt;
    TRY(lt.alloc(ctx, (uint64_t)n1 * N * 8));
    launch_transpose_u64(d_L, N, n1, lt.at<uint64_t>(), N, s);
    launch_gemm_abt(d_mq, lt.at<uint64_t>(), nullptr, rows, n1, N, al_rm.at<uint64_t>(), s);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

int check_plain_inputs(const uint64_t* m_q, uint64_t rows, const uint64_t* L, const uint64_t* H, uint32_t n1,
                       bn_sparse_csr S) {
    if ((rows && (!m_q || !H || !S.rowptr)) || !L) return fail(BN_EINVAL, "null input array");
    TRY(validate_residues(m_q, rows * N, "m_q"));
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    TRY(validate_residues(H, rows * n1, "h"));
    if (rows && S.rowptr[rows] && (!S.idx || !S.sign)) return fail(BN_EINVAL, "s_mat arrays are null");
    for (uint64_t e = 0; rows && e < S.rowptr[rows]; ++e)
        if (S.idx[e] >= N || (S.sign[e] != 1 && S.sign[e] != -1)) return fail(BN_EINVAL, "bad s_mat entry %llu", (unsigned long long)e);
    return BN_OK;
}

// Encrypt on device and fill a corpus (server + client state).
int build_corpus_from_plain(bn_ctx* ctx, Corpus& c, const uint64_t* m_q, uint64_t rows, uint32_t n1, const uint64_t* L,
                            const uint64_t* H, bn_sparse_csr S, cudaStream_t s) {
    c.rows = rows;
    c.n1 = n1;
    DevMem d_mq, d_L, d_H, al_rm;
    TRY(d_mq.alloc(ctx, rows * N * 8));
    TRY(d_L.alloc(ctx, (uint64_t)N * n1 * 8));
    TRY(d_H.alloc(ctx, rows * n1 * 8));
    if (rows) {
        CU(cudaMemcpyAsync(d_mq.p, m_q, rows * N * 8, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(d_H.p, H, rows * n1 * 8, cudaMemcpyHostToDevice, s));
    }
    CU(cudaMemcpyAsync(d_L.p, L, (uint64_t)N * n1 * 8, cudaMemcpyHostToDevice, s));
    TRY(device_encrypt(ctx, d_mq.at<uint64_t>(), rows, n1, d_L.at<uint64_t>(), d_H.at<uint64_t>(), S, c.m_enc, al_rm, s));
    TRY(corpus_tmap(c));
    TRY(device_colmajor(ctx, al_rm.at<uint64_t>(), rows, n1, c.al_cm, s));
    TRY(device_colmajor(ctx, d_H.at<uint64_t>(), rows, n1, c.h_cm, s));
    TRY(device_colmajor(ctx, d_mq.at<uint64_t>(), rows, N, c.mp_cm, s));
    CU(cudaStreamSynchronize(s));
    TRY(c.L.alloc(ctx, (uint64_t)N * n1 * 8));
    CU(cudaMemcpyAsync(c.L.p, L, (uint64_t)N * n1 * 8, cudaMemcpyHostToDevice, s));
    TRY(upload_sparse_ell(ctx, S, rows, c, s));
    CU(cudaStreamSynchronize(s));
    TRY(build_decode_layout(ctx, c, s));
    c.client = true;
    return BN_OK;
}

// The sparsity threshold of sample_sparse_pm1 (crypto.rs:207-223): mu 2^32
// in f64, truncated, as the host keygen computes it.
uint32_t sparse_threshold() {
    const double t = bn_host_mu() * 4294967296.0;
    const uint64_t u = t <= 0.0 ? 0 : (uint64_t)t;
    return (uint32_t)std::min<uint64_t>(u, 0xffffffffull);
}

// H and S of one cluster from its h_seed on the device (bn_keygen.cu):
// H -> d_H (rows x n1), S -> d_rowptr (rows + 1, from 0), d_idx / d_sign
// (at most cap entries); *nnz = S's entries.
int device_keygen(bn_ctx* ctx, const uint8_t seed[32], uint64_t rows, uint32_t n1, uint64_t* d_H, uint64_t* d_rowptr,
                  uint32_t* d_idx, int8_t* d_sign, uint64_t cap, DevMem& scratch, DevMem& status, uint64_t* nnz,
                  cudaStream_t s) {
    *nnz = 0;
    if (!rows) return BN_OK;
    TRY(scratch.reserve(ctx, keygen_s_scratch_bytes(rows, N)));
    TRY(status.reserve(ctx, 16));
    CU(cudaMemsetAsync(status.p, 0, 16, s));
    uint32_t* st = status.at<uint32_t>();
    launch_keygen_h(seed, rows * n1, d_H, st + 2, ctx->num_sms, s);
    launch_keygen_s(seed, rows, N, n1, sparse_threshold(), scratch.p, cap, d_idx, d_sign, d_rowptr, st, s);
    CU(cudaGetLastError());
    uint32_t h[3];
    CU(cudaMemcpyAsync(h, st, 12, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(nnz, d_rowptr + rows, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (!h[0] || h[1]) return fail(BN_EINVAL, "S has more entries than the keygen sizes for (m n / 4)");
    if (h[2] & DRAW_HIT_P)
        return fail(BN_EDRAW, "an H draw equalled p (regenerate_h_s redraws there, crypto.rs:155-162); draw this "
                              "cluster's keys on the host (bn_host_regenerate_h_s)");
    return BN_OK;
}

// Corpus from the plaintext with H and S already on the device: encryption,
// client arrays and decode layouts (the device-resident form of
// build_corpus_from_plain).
int build_corpus_device_keys(bn_ctx* ctx, Corpus& c, const uint64_t* m_q, uint64_t rows, uint32_t n1,
                             const uint64_t* L, DevMem& d_H, const uint64_t* h_rowptr, DevMem& d_rowptr, DevMem& d_idx,
                             DevMem& d_sign, cudaStream_t s) {
    c.rows = rows;
    c.n1 = n1;
    DevMem d_mq, d_L, al_rm;
    TRY(d_mq.alloc(ctx, rows * N * 8));
    TRY(d_L.alloc(ctx, (uint64_t)N * n1 * 8));
    if (rows) CU(cudaMemcpyAsync(d_mq.p, m_q, rows * N * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(d_L.p, L, (uint64_t)N * n1 * 8, cudaMemcpyHostToDevice, s));
    TRY(device_encrypt_dev(ctx, d_mq.at<uint64_t>(), rows, n1, d_L.at<uint64_t>(), d_H.at<uint64_t>(),
                           d_rowptr.at<uint64_t>(), d_idx.at<uint32_t>(), d_sign.at<int8_t>(), c.m_enc, al_rm, s));
    TRY(corpus_tmap(c));
    TRY(device_colmajor(ctx, al_rm.at<uint64_t>(), rows, n1, c.al_cm, s));
    TRY(device_colmajor(ctx, d_H.at<uint64_t>(), rows, n1, c.h_cm, s));
    TRY(device_colmajor(ctx, d_mq.at<uint64_t>(), rows, N, c.mp_cm, s));
    CU(cudaStreamSynchronize(s));
    TRY(c.L.alloc(ctx, (uint64_t)N * n1 * 8));
    CU(cudaMemcpyAsync(c.L.p, L, (uint64_t)N * n1 * 8, cudaMemcpyHostToDevice, s));
    TRY(ell_from_device_csr(ctx, h_rowptr, d_rowptr.at<uint64_t>(), d_idx.at<uint32_t>(), d_sign.at<int8_t>(), rows, c,
                            s));
    TRY(build_decode_layout(ctx, c, s));
    c.client = true;
    return BN_OK;
}

// Keys of `lists` clusters (list c owns rows [off[c], off[c+1]) and has
// seed seeds[c]) drawn on the device into one H and one concatenated CSR.
int keygen_lists(bn_ctx* ctx, uint32_t lists, const uint64_t* off, const uint8_t* seeds, uint32_t n1, DevMem& H,
                 DevMem& rowptr, DevMem& idx, DevMem& sign, std::vector<uint64_t>& h_rowptr, cudaStream_t s) {
    const uint64_t rows = off[lists];
    const uint64_t cap = rows * N / 4 + 1024;
    TRY(H.alloc(ctx, std::max<uint64_t>(rows * n1, 1) * 8));
    TRY(rowptr.alloc(ctx, (rows + 1) * 8));
    TRY(idx.alloc(ctx, cap * 4));
    TRY(sign.alloc(ctx, cap));
    DevMem scratch, status, local;
    uint64_t base = 0, max_rows = 0;
    for (uint32_t c = 0; c < lists; ++c) max_rows = std::max(max_rows, off[c + 1] - off[c]);
    TRY(local.alloc(ctx, (max_rows + 1) * 8));
    CU(cudaMemsetAsync(rowptr.p, 0, 8, s));
    for (uint32_t c = 0; c < lists; ++c) {
        const uint64_t o = off[c], m = off[c + 1] - o;
        if (!m) continue;
        uint64_t nnz = 0;
        TRY(device_keygen(ctx, seeds + 32ull * c, m, n1, H.at<uint64_t>() + o * n1, local.at<uint64_t>(),
                          idx.at<uint32_t>() + base, sign.at<int8_t>() + base, cap - base, scratch, status, &nnz, s));
        launch_rowptr_shift(local.at<uint64_t>(), m + 1, base, rowptr.at<uint64_t>() + o, s);
        base += nnz;
    }
    CU(cudaGetLastError());
    h_rowptr.resize(rows + 1);
    CU(cudaMemcpyAsync(h_rowptr.data(), rowptr.p, (rows + 1) * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

// ------------------------------------------------------------------ pipeline
void finish_meta(HostMeta& hm) {
    hm.seg_blk.assign(hm.segs.size() + 1, 0);
    hm.seg_unit.assign(hm.segs.size() + 1, 0);
    for (size_t i = 0; i < hm.segs.size(); ++i) {
        const ScanSeg& sg = hm.segs[i];
        hm.seg_blk[i + 1] = hm.seg_blk[i] + (sg.rows + SCAN_ROWS - 1) / SCAN_ROWS;
        hm.seg_unit[i + 1] = hm.seg_unit[i] + (sg.rows ? ((sg.row0 + sg.rows - 1) >> 5) - (sg.row0 >> 5) + 1 : 0);
    }
    hm.blocks.clear();
    hm.panels.clear();
    hm.seg_block0.assign(hm.vsegs.size() + 1, 0);
    hm.seg_panel0.assign(hm.vsegs.size() + 1, 0);
    for (uint32_t s = 0; s < hm.vsegs.size(); ++s) {
        const VerifySeg& v = hm.vsegs[s];
        hm.seg_block0[s] = (uint32_t)hm.blocks.size();
        hm.seg_panel0[s] = (uint32_t)hm.panels.size();
        for (uint32_t i0 = 0; i0 < v.rows; i0 += TC_ROWS) hm.blocks.push_back(TcBlock{s, i0});
        for (uint32_t p0 = 0; p0 < v.rows; p0 += TC_PANEL_ROWS)
            hm.panels.push_back(TcPanel{v.row0 + p0, std::min<uint32_t>(TC_PANEL_ROWS, v.rows - p0),
                                        hm.seg_block0[s] + p0 / TC_ROWS, s, 0});
    }
    hm.seg_block0.back() = (uint32_t)hm.blocks.size();
    hm.seg_panel0.back() = (uint32_t)hm.panels.size();
}

void flat_meta(uint64_t m, uint32_t B, HostMeta& hm) {
    hm = HostMeta();
    for (uint32_t b = 0; b < B; ++b) {
        hm.segs.push_back(ScanSeg{0, (uint64_t)b * m, (uint32_t)m, b});
        hm.vsegs.push_back(VerifySeg{0, (uint64_t)b * m, (uint32_t)m, b});
        hm.dq.push_back(DecodeQuery{b, 1});
    }
    hm.total_out = (uint64_t)B * m;
    hm.max_rows = m;
    finish_meta(hm);
}

int pick_ctas(uint64_t max_rows_per_query, uint32_t B, int sms) {
    uint64_t by_rows = (max_rows_per_query + 255) / 256;
    uint64_t by_sms = std::max<uint64_t>(1, (uint64_t)sms * 4 / std::max<uint32_t>(B, 1));
    return (int)std::max<uint64_t>(1, std::min(by_rows, by_sms));
}

RunLayout make_layout(const Sizes& z, bool want_mv) {
    Layout L;
    RunLayout o{};
    o.v = L.take<uint64_t>((uint64_t)z.B * N);
    o.g = L.take<uint64_t>((uint64_t)z.B * z.n1);
    o.t = L.take<uint32_t>((uint64_t)z.B * N);
    o.t_nnz = L.take<uint32_t>(z.B);
    o.seeds = L.take<uint8_t>((uint64_t)z.B * 32);
    o.segs = L.take<ScanSeg>(z.nseg);
    o.seg_blk = L.take<uint64_t>(z.nseg + 1);
    o.seg_unit = L.take<uint64_t>(z.nseg + 1);
    o.vsegs = L.take<VerifySeg>(z.nvseg);
    o.dq = L.take<DecodeQuery>(z.B);
    o.tc_blocks = L.take<TcBlock>(z.nblocks);
    o.tc_panels = L.take<TcPanel>(z.npanels);
    o.seg_panel0 = L.take<uint32_t>(z.nvseg + 1);
    o.seg_block0 = L.take<uint32_t>(z.nvseg + 1);
    o.in_end = L.off;
    o.ids = L.take<uint32_t>((uint64_t)z.B * std::max<uint32_t>(z.k, 1));
    o.out_begin = o.ids;
    o.scores = L.take<int64_t>((uint64_t)z.B * std::max<uint32_t>(z.k, 1));
    o.n = L.take<uint32_t>(z.B);
    o.vfailed = L.take<int32_t>(std::max<uint64_t>(z.nvseg, 1));
    o.ur = L.take<uint64_t>(std::max<uint64_t>(z.nvseg * z.trials, 1));
    o.zv = L.take<uint64_t>(std::max<uint64_t>(z.nvseg * z.trials, 1));
    o.err = L.take<uint32_t>(1);
    o.flags = L.take<uint32_t>(1);  // DRAW_HIT_P when a Protocol 2 draw equalled p
    o.out_end = L.off;
    o.limbs = L.take<QLimb>((uint64_t)z.B * N);
    o.x = L.take<uint64_t>((uint64_t)z.B * z.n1);
    o.r = L.take<uint64_t>(std::max<uint64_t>(z.total_out, 1));
    o.mv = want_mv ? L.take<uint64_t>(std::max<uint64_t>(z.total_out, 1)) : 0;
    const bool tc = z.engine == BN_ENGINE_TENSOR;
    const uint64_t zp = !z.trials ? 1 : tc ? z.npanels * z.trials * N : (uint64_t)z.nvseg * z.fp.chunks * z.trials * N;
    const uint64_t up = !z.trials ? 1 : tc ? z.nblocks * z.trials : (uint64_t)z.nvseg * z.fp.chunks * z.trials;
    o.z_part = L.take<uint64_t>(std::max<uint64_t>(zp, 1));
    o.ur_part = L.take<uint64_t>(std::max<uint64_t>(up, 1));
    const uint64_t cand = (uint64_t)z.ctas * std::max<uint32_t>(z.k, 1);  // z.ctas: decode CTAs of all queries
    o.cand_s = L.take<int64_t>(cand);
    o.cand_i = L.take<uint32_t>(cand);
    o.cand_n = L.take<uint32_t>(z.ctas);
    o.cand_done = L.take<uint32_t>(z.B);
    o.u_buf = (tc && z.trials) ? L.take<uint8_t>(std::max<uint64_t>(z.nblocks, 1) * pass_rows(TC_MAX_TRIALS) * TC_ROWS) : 0;
    o.r_part = (tc && z.trials)
                   ? L.take<uint64_t>((uint64_t)tc_groups(pass_rows(std::min<uint32_t>(TC_MAX_TRIALS, z.trials))) *
                                      std::max<uint64_t>(z.total_out, 1))
                   : 0;
    o.zv_chunks = L.take<uint64_t>(std::max<uint64_t>(tc_finish_words((uint32_t)z.nvseg, z.trials), 1));
    o.wimg = (tc && z.trials) ? L.take<uint8_t>((uint64_t)z.B * WIMG_BYTES_PER_QUERY) : 0;
    o.total = L.off + 1024;
    return o;
}

int make_tc_maps(const Sizes& z, const uint8_t* d_u, const uint8_t* d_w, TcMaps& maps) {
    if (z.engine != BN_ENGINE_TENSOR || !z.trials || !z.nblocks) return BN_OK;
    {
        cudaError_t e = make_tmap_u8(&maps.w, d_w, 128, (uint64_t)z.B * 64 * 16, 128, WIMG_BOX_ROWS);
        if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map for the query images: %s", cudaGetErrorString(e));
    }
    for (uint32_t t0 = 0, ps = 0; t0 < z.trials; t0 += TC_MAX_TRIALS, ++ps) {
        const uint32_t nr = pass_rows(std::min<uint32_t>(TC_MAX_TRIALS, z.trials - t0));
        cudaError_t e = make_tmap_u8(&maps.u[ps], d_u, TC_ROWS, z.nblocks * (uint64_t)nr, TC_ROWS, nr);
        if (e != cudaSuccess) return fail(BN_ECUDA, "tensor map for the Freivalds draws: %s", cudaGetErrorString(e));
    }
    return BN_OK;
}

// prof0 / prof1 (nullable): events recorded on s right before and after the
// pipeline's dominant kernel, the single pass over m_enc (fused scan +
// Protocol 2 on the tensor engine, else the scan).
int enqueue_pipeline(bn_ctx* ctx, const Corpus& c, const Sizes& z, const Meta& m, const Inputs& in, const Scratch& sc,
                     const Outputs& out, cudaStream_t s, cudaEvent_t prof0, cudaEvent_t prof1) {
    CU(cudaMemsetAsync(sc.err, 0, 4, s));
    CU(cudaMemsetAsync(sc.flags, 0, 4, s));
    if (z.trials && ctx->debug_draw_hit) launch_or_flag(sc.flags, DRAW_HIT_P, s);
    launch_query_limbs(in.v, z.B, sc.limbs, s);
    const ChaChaKey* keys = reinterpret_cast<const ChaChaKey*>(in.seeds);
    if (z.trials && z.engine == BN_ENGINE_TENSOR) {
        // One pass over m_enc yields r and the first <= 20 trials' z (tensor
        // cores); later passes of 20 trials reuse the now-known r.
        for (uint32_t t0 = 0, ps = 0; t0 < z.trials; t0 += TC_MAX_TRIALS, ++ps) {
            const uint32_t tc = std::min<uint32_t>(TC_MAX_TRIALS, z.trials - t0), nr = pass_rows(tc);
            if (ps == 0) {
                launch_tc_ugen(m.vsegs, m.tc_blocks, m.nblocks, keys, nullptr, t0, tc, nr, sc.u_buf, sc.ur_part,
                               z.trials, sc.flags, s);
                launch_query_wimg(in.v, z.B, sc.wimg, s);
                if (prof0) CU(cudaEventRecord(prof0, s));
                launch_tc_fused(c.tmap_m, m.maps->u[ps], m.maps->w, m.tc_panels, m.npanels, m.vsegs, tc, nr,
                                z.trials, sc.z_part, sc.r_part, z.total_out, sc.err, ctx->num_sms, s,
                                ctx->debug_wait_cycles);
                if (prof1) CU(cudaEventRecord(prof1, s));
                launch_tc_rreduce(m.vsegs, m.tc_blocks, m.nblocks, sc.r_part, z.total_out, tc_groups(nr), sc.u_buf, tc,
                                  nr, z.trials, sc.r, sc.ur_part, s);
            } else {
                launch_tc_ugen(m.vsegs, m.tc_blocks, m.nblocks, keys, sc.r, t0, tc, nr, sc.u_buf, sc.ur_part, z.trials,
                               sc.flags, s);
                launch_tc_freivalds(c.tmap_m, m.maps->u[ps], m.tc_panels, m.npanels, t0, tc, nr, z.trials, sc.z_part,
                                    sc.err, ctx->num_sms, s, 0, ctx->debug_wait_cycles);
            }
        }
        launch_tc_finish(sc.z_part, sc.ur_part, m.seg_panel0, m.seg_block0, in.v, m.vsegs, m.nvseg, z.trials, sc.ur,
                         sc.zv, sc.zv_chunks, out.vfailed, s);
    } else {
        if (prof0) CU(cudaEventRecord(prof0, s));
        launch_scan(c.m_enc.at<uint64_t>(), sc.limbs, m.segs, m.seg_blk, m.nseg, m.total_blocks, sc.r, ctx->num_sms,
                    sc.err, s, ctx->debug_wait_cycles);
        if (prof1) CU(cudaEventRecord(prof1, s));
        if (z.trials) {
            launch_freivalds(c.m_enc.at<uint64_t>(), sc.r, m.vsegs, m.nvseg, keys, z.trials, z.fp, sc.z_part, sc.ur_part,
                             sc.flags, s);
            launch_freivalds_finish(sc.z_part, sc.ur_part, in.v, m.vsegs, m.nvseg, z.trials, z.fp, sc.ur, sc.zv,
                                    out.vfailed, s);
        } else {
            CU(cudaMemsetAsync(out.vfailed, 0xff, std::max<uint64_t>(m.nvseg, 1) * 4, s));
        }
    }
    if (z.k) {
        launch_lt_times_v(c.L.at<uint64_t>(), c.n1, in.v, z.B, sc.x, s);
        launch_decode_topk(sc.r, decode_corpus(c), m.segs, m.seg_unit, m.dq, z.B, in.v, in.g, sc.x, in.t, in.t_nnz, z.k,
                           z.ctas, sc.topk, out.mv, out.ids, out.scores, out.n, s);
    } else {
        CU(cudaMemsetAsync(out.n, 0, (uint64_t)z.B * 4, s));
    }
    CU(cudaGetLastError());
    return BN_OK;
}

Meta meta_at(char* d, const RunLayout& o, const HostMeta& hm, const TcMaps* maps) {
    return Meta{reinterpret_cast<ScanSeg*>(d + o.segs), reinterpret_cast<uint64_t*>(d + o.seg_blk),
                reinterpret_cast<uint64_t*>(d + o.seg_unit), (uint32_t)hm.segs.size(), hm.seg_blk.empty() ? 0 : hm.seg_blk.back(),
                reinterpret_cast<VerifySeg*>(d + o.vsegs), (uint32_t)hm.vsegs.size(),
                reinterpret_cast<DecodeQuery*>(d + o.dq), reinterpret_cast<TcBlock*>(d + o.tc_blocks),
                (uint32_t)hm.blocks.size(), reinterpret_cast<TcPanel*>(d + o.tc_panels), (uint32_t)hm.panels.size(),
                reinterpret_cast<uint32_t*>(d + o.seg_panel0), reinterpret_cast<uint32_t*>(d + o.seg_block0), maps};
}
Scratch scratch_at(char* d, const RunLayout& o) {
    return Scratch{reinterpret_cast<QLimb*>(d + o.limbs), reinterpret_cast<uint64_t*>(d + o.x),
                   reinterpret_cast<uint64_t*>(d + o.r), reinterpret_cast<uint64_t*>(d + o.z_part),
                   reinterpret_cast<uint64_t*>(d + o.ur_part), reinterpret_cast<uint32_t*>(d + o.flags),
                   reinterpret_cast<uint64_t*>(d + o.ur), reinterpret_cast<uint64_t*>(d + o.zv),
                   TopkScratch{reinterpret_cast<int64_t*>(d + o.cand_s), reinterpret_cast<uint32_t*>(d + o.cand_i),
                               reinterpret_cast<uint32_t*>(d + o.cand_n), reinterpret_cast<uint32_t*>(d + o.cand_done)},
                   reinterpret_cast<uint32_t*>(d + o.err), reinterpret_cast<uint8_t*>(d + o.u_buf),
                   reinterpret_cast<uint64_t*>(d + o.r_part), reinterpret_cast<uint64_t*>(d + o.zv_chunks),
                   reinterpret_cast<uint8_t*>(d + o.wimg)};
}
void pack_meta(char* h, const RunLayout& o, const HostMeta& hm) {
    memcpy(h + o.segs, hm.segs.data(), hm.segs.size() * sizeof(ScanSeg));
    memcpy(h + o.seg_blk, hm.seg_blk.data(), hm.seg_blk.size() * 8);
    memcpy(h + o.seg_unit, hm.seg_unit.data(), hm.seg_unit.size() * 8);
    memcpy(h + o.vsegs, hm.vsegs.data(), hm.vsegs.size() * sizeof(VerifySeg));
    memcpy(h + o.dq, hm.dq.data(), hm.dq.size() * sizeof(DecodeQuery));
    memcpy(h + o.tc_blocks, hm.blocks.data(), hm.blocks.size() * sizeof(TcBlock));
    memcpy(h + o.tc_panels, hm.panels.data(), hm.panels.size() * sizeof(TcPanel));
    memcpy(h + o.seg_panel0, hm.seg_panel0.data(), hm.seg_panel0.size() * 4);
    memcpy(h + o.seg_block0, hm.seg_block0.data(), hm.seg_block0.size() * 4);
}

int engine_init(Engine& e, bn_ctx* ctx) {
    e.ctx = ctx;
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
    return BN_OK;
}

void engine_free(Engine& e) {
    if (e.stream) {
        cudaStreamSynchronize(e.stream);
        cudaStreamDestroy(e.stream);
    }
}

// Decode CTAs of a run: DECODE_CTAS_PER_SM per SM in total (one wave of
// the decode kernel), shared among the queries in proportion to their
// units (32-row blocks), at least one per query and at most one per tile
// of 8 units.  Returns the total.
uint32_t assign_decode_ctas(HostMeta& hm, int sms) {
    std::vector<uint64_t> units(hm.dq.size(), 0);
    uint64_t total = 0;
    for (size_t q = 0; q < hm.dq.size(); ++q) {
        const DecodeQuery& d = hm.dq[q];
        if (d.nseg) units[q] = hm.seg_unit[d.seg0 + d.nseg] - hm.seg_unit[d.seg0];
        total += units[q];
    }
    const uint64_t target = (uint64_t)sms * DECODE_CTAS_PER_SM;
    uint32_t next = 0;
    for (size_t q = 0; q < hm.dq.size(); ++q) {
        uint64_t c = total ? (target * units[q] + total - 1) / total : 1;
        c = std::max<uint64_t>(1, std::min(c, (units[q] + 7) / 8));
        hm.dq[q].cta0 = next;
        hm.dq[q].ctas = (uint32_t)c;
        next += (uint32_t)c;
    }
    return next;
}

Sizes sizes_for(const Engine& e, HostMeta& hm, uint32_t B, uint32_t trials, uint32_t k) {
    return Sizes{B, e.c.n1, trials, k, assign_decode_ctas(hm, e.ctx->num_sms), hm.total_out,
                 hm.segs.size(), hm.vsegs.size(), hm.blocks.size(), hm.panels.size(),
                 plan_freivalds(std::max<uint64_t>(hm.max_rows, 1), (uint32_t)std::max<size_t>(hm.vsegs.size(), 1),
                                e.ctx->num_sms),
                 e.ctx->engine};
}

// One pipeline run over host inputs, split so that a caller can keep several
// runs in flight on different streams (the serving loop): prepare packs the
// inputs into pinned staging, launch enqueues H2D + pipeline + D2H, finish
// reads the outputs once the stream has drained.
int job_prepare(Engine& e, QueryJob& j, DevMem& ws, PinnedMem& host, const uint64_t* v_enc, const uint64_t* g,
                const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds) {
    Corpus& c = e.c;
    HostMeta& hm = *j.hm;
    const uint32_t B = j.B, trials = j.trials, k = j.k;
    if (!c.client) return fail(BN_EUNSUPPORTED, "this handle has no client state (attach_client was not called)");
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX = %d", k, BN_TOPK_MAX);
    if (B > 65535) return fail(BN_EINVAL, "B = %u exceeds 65535 queries per call", B);
    if (trials > MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %u", trials, MAX_TRIALS);
    if (trials && !v_seeds) return fail(BN_EINVAL, "v_seeds is required when trials > 0");
    if (!v_enc || !g || !t_nnz) return fail(BN_EINVAL, "null query input");
    uint64_t t_total = 0;
    for (uint32_t b = 0; b < B; ++b) {
        if (t_nnz[b] > N) return fail(BN_EINVAL, "t_nnz[%u] = %u exceeds n", b, t_nnz[b]);
        t_total += t_nnz[b];
    }
    if (t_total && (!t_idx || !t_sign)) return fail(BN_EINVAL, "t_idx / t_sign are null");
    TRY(validate_residues(v_enc, (uint64_t)B * N, "v_enc"));
    TRY(validate_residues(g, (uint64_t)B * c.n1, "g"));

    j.z = sizes_for(e, hm, B, trials, k);
    j.o = make_layout(j.z, j.want_mv);
    const RunLayout& o = j.o;
    TRY(ws.reserve_grow(e.ctx, o.total));
    TRY(host.reserve(o.out_end));
    char* d = ws.at<char>();
    TRY(make_tc_maps(j.z, reinterpret_cast<uint8_t*>(d + o.u_buf), reinterpret_cast<uint8_t*>(d + o.wimg), j.maps));

    char* h = host.at<char>();
    memcpy(h + o.v, v_enc, (uint64_t)B * N * 8);
    memcpy(h + o.g, g, (uint64_t)B * c.n1 * 8);
    uint32_t* ht = reinterpret_cast<uint32_t*>(h + o.t);
    uint64_t tp = 0;
    for (uint32_t b = 0; b < B; ++b) {
        for (uint32_t i = 0; i < t_nnz[b]; ++i, ++tp) {
            if (t_idx[tp] >= N || (t_sign[tp] != 1 && t_sign[tp] != -1))
                return fail(BN_EINVAL, "T entry %llu is not (col < n, sign +-1)", (unsigned long long)tp);
            ht[(uint64_t)b * N + i] = t_idx[tp] | (t_sign[tp] < 0 ? 0x80000000u : 0u);
        }
    }
    memcpy(h + o.t_nnz, t_nnz, (uint64_t)B * 4);
    if (v_seeds) memcpy(h + o.seeds, v_seeds, (uint64_t)B * 32);
    else memset(h + o.seeds, 0, (uint64_t)B * 32);
    pack_meta(h, o, hm);
    return BN_OK;
}

int job_launch(Engine& e, QueryJob& j, DevMem& ws, PinnedMem& host, cudaStream_t s, uint64_t* r_out, uint64_t* mv_out) {
    const HostMeta& hm = *j.hm;
    const RunLayout& o = j.o;
    char* d = ws.at<char>();
    char* h = host.at<char>();
    CU(cudaSetDevice(e.ctx->device));
    CU(cudaMemcpyAsync(d, h, o.in_end, cudaMemcpyHostToDevice, s));
    const Meta m = meta_at(d, o, hm, &j.maps);
    Inputs in{reinterpret_cast<uint64_t*>(d + o.v), reinterpret_cast<uint64_t*>(d + o.g),
              reinterpret_cast<uint32_t*>(d + o.t), reinterpret_cast<uint32_t*>(d + o.t_nnz),
              reinterpret_cast<uint8_t*>(d + o.seeds)};
    const Scratch sc = scratch_at(d, o);
    Outputs out{reinterpret_cast<uint32_t*>(d + o.ids), reinterpret_cast<int64_t*>(d + o.scores),
                reinterpret_cast<uint32_t*>(d + o.n), reinterpret_cast<int32_t*>(d + o.vfailed),
                j.want_mv ? reinterpret_cast<uint64_t*>(d + o.mv) : nullptr};
    if (hm.segs.empty()) {
        CU(cudaMemsetAsync(out.n, 0, (uint64_t)j.B * 4, s));
        CU(cudaMemsetAsync(sc.err, 0, 4, s));
        CU(cudaMemsetAsync(sc.flags, 0, 4, s));
    } else {
        TRY(enqueue_pipeline(e.ctx, e.c, j.z, m, in, sc, out, s, nullptr, nullptr));
    }
    CU(cudaMemcpyAsync(h + o.out_begin, d + o.out_begin, o.out_end - o.out_begin, cudaMemcpyDeviceToHost, s));
    if (r_out && hm.total_out) CU(cudaMemcpyAsync(r_out, d + o.r, hm.total_out * 8, cudaMemcpyDeviceToHost, s));
    if (mv_out && hm.total_out) CU(cudaMemcpyAsync(mv_out, d + o.mv, hm.total_out * 8, cudaMemcpyDeviceToHost, s));
    return BN_OK;
}

int job_finish(const QueryJob& j, const PinnedMem& host, uint32_t* ids, int64_t* scores, uint32_t* n_hits,
               std::vector<int32_t>& vfailed) {
    const HostMeta& hm = *j.hm;
    const RunLayout& o = j.o;
    const char* h = host.at<char>();
    TRY(device_flags_status(*reinterpret_cast<const uint32_t*>(h + o.err) |
                            *reinterpret_cast<const uint32_t*>(h + o.flags)));
    const uint32_t k = j.k, ks = std::max<uint32_t>(k, 1);
    const uint32_t* hid = reinterpret_cast<const uint32_t*>(h + o.ids);
    const int64_t* hsc = reinterpret_cast<const int64_t*>(h + o.scores);
    const uint32_t* hn = reinterpret_cast<const uint32_t*>(h + o.n);
    for (uint32_t b = 0; b < j.B; ++b) {
        const uint32_t nh = hm.segs.empty() ? 0 : hn[b];
        if (n_hits) n_hits[b] = nh;
        if (k) {
            if (ids) memcpy(ids + (uint64_t)b * k, hid + (uint64_t)b * ks, (uint64_t)nh * 4);
            if (scores) memcpy(scores + (uint64_t)b * k, hsc + (uint64_t)b * ks, (uint64_t)nh * 8);
        }
    }
    vfailed.assign(hm.vsegs.size(), -1);
    if (!hm.vsegs.empty()) memcpy(vfailed.data(), h + o.vfailed, hm.vsegs.size() * 4);
    return BN_OK;
}

// Host-buffer query: pack, one H2D, pipeline, one D2H, sync.
int run_query(Engine& e, HostMeta& hm, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
              const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
              uint32_t* ids, int64_t* scores, uint32_t* n_hits, std::vector<int32_t>& vfailed, uint64_t* r_out,
              uint64_t* mv_out) {
    QueryJob j;
    j.hm = &hm;
    j.B = B;
    j.trials = trials;
    j.k = k;
    j.want_mv = mv_out != nullptr;
    TRY(job_prepare(e, j, e.ws, e.host, v_enc, g, t_idx, t_sign, t_nnz, v_seeds));
    TRY(job_launch(e, j, e.ws, e.host, e.stream, r_out, mv_out));
    CU(cudaStreamSynchronize(e.stream));
    return job_finish(j, e.host, ids, scores, n_hits, vfailed);
}

// Verify a claimed r for one contiguous row range (Protocol 2 only).
int run_verify(Engine& e, uint64_t row0, uint64_t rows, const uint64_t* r, const uint64_t* v_enc, const uint8_t* seed,
               uint32_t trials, int32_t* failed_trial, uint64_t* ur, uint64_t* zv) {
    if (!failed_trial || !v_enc || !seed || (rows && !r)) return fail(BN_EINVAL, "null argument");
    if (trials > MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %u", trials, MAX_TRIALS);
    TRY(validate_residues(r, rows, "r"));
    TRY(validate_residues(v_enc, N, "v_enc"));
    if (trials == 0 || rows == 0) {
        // the reference's loop body never runs: every (zero) trial passes;
        // with m = 0 both sides are the empty sum.
        *failed_trial = -1;
        for (uint32_t t = 0; t < trials; ++t) { if (ur) ur[t] = 0; if (zv) zv[t] = 0; }
        return BN_OK;
    }
    HostMeta hm;
    hm.vsegs.push_back(VerifySeg{row0, 0, (uint32_t)rows, 0});
    hm.max_rows = rows;
    finish_meta(hm);
    Sizes z{1, e.c.n1, trials, 0, 1, rows, 0, 1, hm.blocks.size(), hm.panels.size(),
            plan_freivalds(rows, 1, e.ctx->num_sms), e.ctx->engine};
    const RunLayout o = make_layout(z, false);
    TRY(e.ws.reserve(e.ctx, o.total));
    TRY(e.host.reserve(o.out_end));
    char* h = e.host.at<char>();
    char* d = e.ws.at<char>();
    TcMaps maps;
    TRY(make_tc_maps(z, reinterpret_cast<uint8_t*>(d + o.u_buf), reinterpret_cast<uint8_t*>(d + o.wimg), maps));
    memcpy(h + o.v, v_enc, N * 8);
    memcpy(h + o.seeds, seed, 32);
    pack_meta(h, o, hm);
    CU(cudaSetDevice(e.ctx->device));
    CU(cudaMemcpyAsync(d, h, o.in_end, cudaMemcpyHostToDevice, e.stream));
    CU(cudaMemcpyAsync(d + o.r, r, rows * 8, cudaMemcpyHostToDevice, e.stream));
    const Meta m = meta_at(d, o, hm, &maps);
    const Scratch sc = scratch_at(d, o);
    const ChaChaKey* keys = reinterpret_cast<const ChaChaKey*>(d + o.seeds);
    const uint64_t* dv = reinterpret_cast<uint64_t*>(d + o.v);
    int32_t* dfail = reinterpret_cast<int32_t*>(d + o.vfailed);
    CU(cudaMemsetAsync(sc.flags, 0, 4, e.stream));
    CU(cudaMemsetAsync(sc.err, 0, 4, e.stream));
    if (e.ctx->debug_draw_hit) launch_or_flag(sc.flags, DRAW_HIT_P, e.stream);
    if (z.engine == BN_ENGINE_TENSOR) {
        for (uint32_t t0 = 0, ps = 0; t0 < trials; t0 += TC_MAX_TRIALS, ++ps) {
            const uint32_t tc = std::min<uint32_t>(TC_MAX_TRIALS, trials - t0), nr = pass_rows(tc);
            launch_tc_ugen(m.vsegs, m.tc_blocks, m.nblocks, keys, sc.r, t0, tc, nr, sc.u_buf, sc.ur_part, trials,
                           sc.flags, e.stream);
            launch_tc_freivalds(e.c.tmap_m, maps.u[ps], m.tc_panels, m.npanels, t0, tc, nr, trials, sc.z_part, sc.err,
                                e.ctx->num_sms, e.stream, 0, e.ctx->debug_wait_cycles);
        }
        launch_tc_finish(sc.z_part, sc.ur_part, m.seg_panel0, m.seg_block0, dv, m.vsegs, 1, trials, sc.ur, sc.zv,
                         sc.zv_chunks, dfail, e.stream);
    } else {
        launch_freivalds(e.c.m_enc.at<uint64_t>(), sc.r, m.vsegs, 1, keys, trials, z.fp, sc.z_part, sc.ur_part, sc.flags,
                         e.stream);
        launch_freivalds_finish(sc.z_part, sc.ur_part, dv, m.vsegs, 1, trials, z.fp, sc.ur, sc.zv, dfail, e.stream);
    }
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h + o.out_begin, d + o.out_begin, o.out_end - o.out_begin, cudaMemcpyDeviceToHost, e.stream));
    CU(cudaStreamSynchronize(e.stream));
    TRY(device_flags_status(*reinterpret_cast<const uint32_t*>(h + o.err) |
                            *reinterpret_cast<const uint32_t*>(h + o.flags)));
    *failed_trial = *reinterpret_cast<int32_t*>(h + o.vfailed);
    const uint32_t ran = *failed_trial < 0 ? trials : (uint32_t)*failed_trial + 1;
    for (uint32_t t = 0; t < trials; ++t) {
        if (ur) ur[t] = t < ran ? reinterpret_cast<uint64_t*>(h + o.ur)[t] : 0;
        if (zv) zv[t] = t < ran ? reinterpret_cast<uint64_t*>(h + o.zv)[t] : 0;
    }
    return BN_OK;
}

// Scan rows [row0, row0+rows) against B queries; r is B x rows (host).
int run_scan(Engine& e, uint64_t row0, uint64_t rows, const uint64_t* v_encs, uint32_t B, uint64_t* r) {
    if (!v_encs || (rows && B && !r)) return fail(BN_EINVAL, "null argument");
    TRY(validate_residues(v_encs, (uint64_t)B * N, "v_enc"));
    if (!rows || !B) return BN_OK;
    HostMeta hm;
    for (uint32_t b = 0; b < B; ++b) hm.segs.push_back(ScanSeg{row0, (uint64_t)b * rows, (uint32_t)rows, b});
    finish_meta(hm);
    Layout L;
    const uint64_t o_v = L.take<uint64_t>((uint64_t)B * N), o_s = L.take<ScanSeg>(B), o_b = L.take<uint64_t>(B + 1), in_end = L.off;
    const uint64_t o_l = L.take<QLimb>((uint64_t)B * N), o_r = L.take<uint64_t>((uint64_t)B * rows);
    const uint64_t o_e = L.take<uint32_t>(1);
    TRY(e.ws.reserve(e.ctx, L.off));
    TRY(e.host.reserve(std::max<uint64_t>(in_end, 4)));
    char* h = e.host.at<char>();
    memcpy(h + o_v, v_encs, (uint64_t)B * N * 8);
    memcpy(h + o_s, hm.segs.data(), B * sizeof(ScanSeg));
    memcpy(h + o_b, hm.seg_blk.data(), (B + 1) * 8ull);
    char* d = e.ws.at<char>();
    CU(cudaSetDevice(e.ctx->device));
    CU(cudaMemcpyAsync(d, h, in_end, cudaMemcpyHostToDevice, e.stream));
    CU(cudaMemsetAsync(d + o_e, 0, 4, e.stream));
    launch_query_limbs(reinterpret_cast<uint64_t*>(d + o_v), B, reinterpret_cast<QLimb*>(d + o_l), e.stream);
    launch_scan(e.c.m_enc.at<uint64_t>(), reinterpret_cast<QLimb*>(d + o_l), reinterpret_cast<ScanSeg*>(d + o_s),
                reinterpret_cast<uint64_t*>(d + o_b), B, hm.seg_blk.back(), reinterpret_cast<uint64_t*>(d + o_r),
                e.ctx->num_sms, reinterpret_cast<uint32_t*>(d + o_e), e.stream, e.ctx->debug_wait_cycles);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(r, d + o_r, (uint64_t)B * rows * 8, cudaMemcpyDeviceToHost, e.stream));
    uint32_t ev = 0;
    CU(cudaMemcpyAsync(&ev, d + o_e, 4, cudaMemcpyDeviceToHost, e.stream));
    CU(cudaStreamSynchronize(e.stream));
    if (ev) return fail(BN_ECUDA, "a device pipeline wait timed out (flags 0x%x); results discarded", ev);
    return BN_OK;
}

int run_dense_terms(Engine& e, uint64_t row0, uint64_t rows, const uint64_t* g, const uint64_t* lt, uint64_t* out) {
    if (!g || !lt || (rows && !out)) return fail(BN_EINVAL, "null argument");
    TRY(validate_residues(g, e.c.n1, "g"));
    TRY(validate_residues(lt, e.c.n1, "lt_venc"));
    if (!rows) return BN_OK;
    Layout L;
    const uint64_t o_g = L.take<uint64_t>(e.c.n1), o_x = L.take<uint64_t>(e.c.n1), in_end = L.off, o_o = L.take<uint64_t>(rows);
    TRY(e.ws.reserve(e.ctx, L.off));
    TRY(e.host.reserve(in_end));
    char* h = e.host.at<char>();
    memcpy(h + o_g, g, e.c.n1 * 8ull);
    memcpy(h + o_x, lt, e.c.n1 * 8ull);
    char* d = e.ws.at<char>();
    CU(cudaSetDevice(e.ctx->device));
    CU(cudaMemcpyAsync(d, h, in_end, cudaMemcpyHostToDevice, e.stream));
    // column-major arrays: the list's rows are a contiguous slice of each column
    launch_dense_terms(e.c.al_cm.at<uint64_t>() + row0, e.c.h_cm.at<uint64_t>() + row0, rows, e.c.n1,
                       reinterpret_cast<uint64_t*>(d + o_g), reinterpret_cast<uint64_t*>(d + o_x),
                       reinterpret_cast<uint64_t*>(d + o_o), e.stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, d + o_o, rows * 8, cudaMemcpyDeviceToHost, e.stream));
    CU(cudaStreamSynchronize(e.stream));
    return BN_OK;
}

}  // namespace api
}  // namespace bn

// Defined in bn_noalloc.cu: loads the allocation-free verifier's static
// scratch and kernels on `device` and resolves the scratch address.
extern "C" int bn_internal_noalloc_setup(int device);

struct bn_plan {
    bn_flat* h = nullptr;
    Sizes z{};
    RunLayout o{};
    DevMem ws;
    HostMeta hm;
    TcMaps maps;
    BlockPlan* block = nullptr;  // set for block plans (bn_flat_block_plan)
    // kernel timing (bn_plan_profile): event pairs around the dominant kernel
    std::vector<cudaEvent_t> prof;
    uint32_t prof_n = 0;
    ~bn_plan() {
        if (block) block_plan_free(block);
        for (cudaEvent_t e : prof) cudaEventDestroy(e);
    }
};

extern "C" {

const char* bn_last_error(void) { return g_err.c_str(); }

const char* bn_build_info(void) {
    static char buf[256];
    snprintf(buf, sizeof buf, "bn_b200 abi=%d arch=sm_100a cuda=%d.%d n=%u", BN_ABI_VERSION, CUDART_VERSION / 1000,
             (CUDART_VERSION % 1000) / 10, N);
    return buf;
}

int bn_device_count(int* out) {
    if (!out) return fail(BN_EINVAL, "null out");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *out = n;
    return BN_OK;
}

int bn_ctx_create(int device, uint64_t vram_budget_bytes, bn_ctx** out) {
    if (!out) return fail(BN_EINVAL, "null out");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(BN_ENODEV, "no CUDA device is visible");
    }
    if (device < 0 || device >= count) return fail(BN_EINVAL, "device %d out of range (%d visible)", device, count);
    CU(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(BN_ENODEV, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    // the allocation-free verifier's static scratch and kernels are loaded
    // now, while allocating is still allowed (bn_noalloc.cu)
    TRY(bn_internal_noalloc_setup(device));
    auto* c = new bn_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    c->budget = vram_budget_bytes ? vram_budget_bytes : (uint64_t)(free_b * 0.8);
    *out = c;
    return BN_OK;
}

int bn_ctx_destroy(bn_ctx* ctx) {
    delete ctx;
    return BN_OK;
}

int bn_debug_plant_draw_hit(bn_ctx* ctx, int on) {
    if (!ctx) return fail(BN_EINVAL, "null ctx");
    ctx->debug_draw_hit = on ? 1 : 0;
    return BN_OK;
}

int bn_debug_set_wait_limit(bn_ctx* ctx, uint64_t cycles) {
    if (!ctx) return fail(BN_EINVAL, "null ctx");
    if (cycles > 4000000000ull) return fail(BN_EINVAL, "wait limit %llu cycles exceeds the default", (unsigned long long)cycles);
    ctx->debug_wait_cycles = (long long)cycles;
    return BN_OK;
}

int bn_ctx_set_engine(bn_ctx* ctx, int engine) {
    if (!ctx) return fail(BN_EINVAL, "null ctx");
    if (engine != BN_ENGINE_TENSOR && engine != BN_ENGINE_CUDA_CORE) return fail(BN_EINVAL, "unknown engine %d", engine);
    ctx->engine = engine;
    return BN_OK;
}

int bn_ctx_memory(const bn_ctx* ctx, uint64_t* budget, uint64_t* used, uint64_t* peak) {
    if (!ctx) return fail(BN_EINVAL, "null ctx");
    auto* c = const_cast<bn_ctx*>(ctx);
    std::lock_guard<std::mutex> g(c->mu);
    if (budget) *budget = c->budget;
    if (used) *used = c->used;
    if (peak) *peak = c->peak;
    return BN_OK;
}

// ---------------------------------------------------------------- flat
int bn_flat_build(bn_ctx* ctx, const uint64_t* m_enc, const uint64_t* a_l, const uint64_t* h, uint64_t m, uint32_t n,
                  uint32_t n1, bn_flat** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (m > 0xffffffffull) return fail(BN_EINVAL, "cluster size must fit in u32");
    if (m && (!m_enc || !a_l || !h)) return fail(BN_EINVAL, "null corpus array");
    TRY(validate_residues(m_enc, m * N, "m_enc"));
    TRY(validate_residues(a_l, m * n1, "a_l"));
    TRY(validate_residues(h, m * n1, "h"));
    auto* f = new bn_flat();
    int rc = engine_init(f->e, ctx);
    if (rc == BN_OK) {
        Corpus& c = f->e.c;
        c.rows = m;
        c.n1 = n1;
        f->m = m;
        rc = c.m_enc.alloc(ctx, m * N * 8);
        if (rc == BN_OK && m) {
            cudaError_t er = cudaMemcpyAsync(c.m_enc.p, m_enc, m * N * 8, cudaMemcpyHostToDevice, f->e.stream);
            if (er != cudaSuccess) rc = fail(BN_ECUDA, "upload m_enc: %s", cudaGetErrorString(er));
        }
        if (rc == BN_OK) rc = corpus_tmap(c);
        if (rc == BN_OK) rc = upload_colmajor(ctx, a_l, m, n1, c.al_cm, f->e.stream);
        if (rc == BN_OK) rc = upload_colmajor(ctx, h, m, n1, c.h_cm, f->e.stream);
        if (rc == BN_OK && cudaStreamSynchronize(f->e.stream) != cudaSuccess) rc = fail(BN_ECUDA, "upload sync failed");
    }
    if (rc != BN_OK) {
        engine_free(f->e);
        delete f;
        return rc;
    }
    *out = f;
    return BN_OK;
}

int bn_flat_attach_client(bn_flat* f, const uint64_t* L, const uint64_t* m_plain, bn_sparse_csr s_mat) {
    if (!f) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> g(f->e.mu);
    CU(cudaSetDevice(f->e.ctx->device));
    TRY(validate_residues(m_plain, f->m * N, "m_plain"));
    return attach_client(f->e.ctx, f->e.c, L, m_plain, s_mat, f->e.stream);
}

int bn_flat_build_from_plain(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L,
                             const uint64_t* H, bn_sparse_csr S, bn_flat** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (m > 0xffffffffull) return fail(BN_EINVAL, "cluster size must fit in u32");
    TRY(check_plain_inputs(m_q, m, L, H, n1, S));
    auto* f = new bn_flat();
    int rc = engine_init(f->e, ctx);
    f->m = m;
    if (rc == BN_OK) rc = build_corpus_from_plain(ctx, f->e.c, m_q, m, n1, L, H, S, f->e.stream);
    if (rc != BN_OK) {
        engine_free(f->e);
        delete f;
        return rc;
    }
    *out = f;
    return BN_OK;
}

int bn_flat_destroy(bn_flat* f) {
    if (!f) return BN_OK;
    engine_free(f->e);
    delete f;
    return BN_OK;
}

int bn_flat_info(const bn_flat* f, uint64_t* rows, uint64_t* bytes) {
    if (!f) return fail(BN_EINVAL, "null handle");
    if (rows) *rows = f->m;
    if (bytes) *bytes = f->e.c.bytes();
    return BN_OK;
}

int bn_flat_device_m_enc(const bn_flat* f, const uint64_t** d) {
    if (!f || !d) return fail(BN_EINVAL, "null argument");
    *d = f->e.c.m_enc.at<uint64_t>();
    return BN_OK;
}

int bn_flat_compute_products(bn_flat* f, const uint64_t* v_enc, uint64_t* r) {
    return bn_flat_compute_products_batch(f, v_enc, 1, r);
}

int bn_flat_compute_products_batch(bn_flat* f, const uint64_t* v_encs, uint32_t B, uint64_t* r) {
    if (!f) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> g(f->e.mu);
    return run_scan(f->e, 0, f->m, v_encs, B, r);
}

int bn_flat_decode_dense_terms(bn_flat* f, const uint64_t* g, const uint64_t* lt, uint64_t* out) {
    if (!f) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> gd(f->e.mu);
    return run_dense_terms(f->e, 0, f->m, g, lt, out);
}

int bn_flat_verify(bn_flat* f, const uint64_t* r, const uint64_t* v_enc, const uint8_t v_seed[32], uint32_t trials,
                   int32_t* failed_trial, uint64_t* ur, uint64_t* zv) {
    if (!f) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> g(f->e.mu);
    return run_verify(f->e, 0, f->m, r, v_enc, v_seed, trials, failed_trial, ur, zv);
}

int bn_flat_query(bn_flat* f, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                  const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials, uint32_t k,
                  uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial, uint64_t* r_out,
                  uint64_t* mv_out) {
    if (!f) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    std::lock_guard<std::mutex> gd(f->e.mu);
    HostMeta& hm = f->query_meta;  // reused while B stays the same
    if (f->query_meta_B != B) {
        f->query_meta_B = 0;
        hm = HostMeta();
        if (f->m) flat_meta(f->m, B, hm);
        else {
            for (uint32_t b = 0; b < B; ++b) hm.dq.push_back(DecodeQuery{0, 0});
            finish_meta(hm);
        }
        f->query_meta_B = B;
    }
    std::vector<int32_t> vf;
    TRY(run_query(f->e, hm, B, v_enc, g, t_idx, t_sign, t_nnz, v_seeds, trials, k, ids, scores, n_hits, vf, r_out, mv_out));
    if (failed_trial)
        for (uint32_t b = 0; b < B; ++b) failed_trial[b] = f->m ? vf[b] : -1;
    return BN_OK;
}

int bn_flat_query_shard(bn_flat* f, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                        const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds, uint32_t trials,
                        uint32_t k, uint64_t shard_row0, uint64_t total_rows, uint32_t* ids, int64_t* scores,
                        uint32_t* n_hits, uint64_t* ur, uint64_t* zv) {
    if (!f) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (!f->m) return fail(BN_EINVAL, "empty shard");
    if (shard_row0 > total_rows || f->m > total_rows - shard_row0)
        return fail(BN_EINVAL, "shard rows [%llu, %llu) exceed the corpus of %llu rows", (unsigned long long)shard_row0,
                    (unsigned long long)(shard_row0 + f->m), (unsigned long long)total_rows);
    if (shard_row0 + f->m > 0xffffffffull) return fail(BN_EINVAL, "global row ids must fit in u32");
    if (trials && (!ur || !zv)) return fail(BN_EINVAL, "ur / zv are required when trials > 0");
    std::lock_guard<std::mutex> gd(f->e.mu);
    HostMeta hm;
    flat_meta(f->m, B, hm);
    for (VerifySeg& vs : hm.vsegs) {  // draw positions of these rows within the whole corpus
        vs.draw_stride = total_rows;
        vs.draw_base = shard_row0;
    }
    QueryJob j;
    j.hm = &hm;
    j.B = B;
    j.trials = trials;
    j.k = k;
    Engine& e = f->e;
    TRY(job_prepare(e, j, e.ws, e.host, v_enc, g, t_idx, t_sign, t_nnz, v_seeds));
    TRY(job_launch(e, j, e.ws, e.host, e.stream, nullptr, nullptr));
    CU(cudaStreamSynchronize(e.stream));
    std::vector<int32_t> vf;  // local verdicts: meaningless for a shard (decided on the sums)
    TRY(job_finish(j, e.host, ids, scores, n_hits, vf));
    if (k && ids)
        for (uint32_t b = 0; b < B; ++b)
            for (uint32_t i = 0; i < (n_hits ? n_hits[b] : std::min<uint64_t>(k, f->m)); ++i)
                ids[(uint64_t)b * k + i] += (uint32_t)shard_row0;
    if (trials) {
        const char* h = e.host.at<char>();
        memcpy(ur, h + j.o.ur, (uint64_t)B * trials * 8);
        memcpy(zv, h + j.o.zv, (uint64_t)B * trials * 8);
    }
    return BN_OK;
}

int bn_flat_plan(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k, bn_plan** out) {
    if (!f || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    if (!B || B > 65535) return fail(BN_EINVAL, "B must be in 1..=65535");
    if (!f->m) return fail(BN_EINVAL, "empty corpus");
    if (k > BN_TOPK_MAX) return fail(BN_EINVAL, "k = %u exceeds BN_TOPK_MAX", k);
    if (trials > MAX_TRIALS) return fail(BN_EINVAL, "trials = %u exceeds %u", trials, MAX_TRIALS);
    if (k && !f->e.c.client) return fail(BN_EUNSUPPORTED, "this handle has no client state");
    std::lock_guard<std::mutex> gd(f->e.mu);
    auto* p = new bn_plan();
    p->h = f;
    flat_meta(f->m, B, p->hm);
    p->z = sizes_for(f->e, p->hm, B, trials, k);
    p->o = make_layout(p->z, false);
    int rc = p->ws.alloc(f->e.ctx, p->o.total);
    if (rc == BN_OK)
        rc = make_tc_maps(p->z, reinterpret_cast<uint8_t*>(p->ws.at<char>() + p->o.u_buf),
                          reinterpret_cast<uint8_t*>(p->ws.at<char>() + p->o.wimg), p->maps);
    if (rc == BN_OK) {
        std::vector<char> h(p->o.in_end, 0);
        pack_meta(h.data(), p->o, p->hm);
        if (cudaMemcpy(p->ws.p, h.data(), p->o.in_end, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(BN_ECUDA, "plan metadata upload failed");
    }
    if (rc != BN_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return BN_OK;
}

int bn_plan_enqueue(bn_plan* p, const uint64_t* d_v, const uint64_t* d_g, const uint32_t* d_t, const uint32_t* d_t_nnz,
                    const uint8_t* d_seeds, uint32_t* d_ids, int64_t* d_scores, uint32_t* d_n, int32_t* d_failed,
                    void* stream) {
    if (!p) return fail(BN_EINVAL, "null plan");
    if (p->block) return fail(BN_EINVAL, "block plan: use bn_plan_enqueue_block");
    if (!d_v || (p->z.k && (!d_g || !d_t || !d_t_nnz || !d_ids || !d_scores || !d_n)) || (p->z.trials && !d_seeds) || !d_failed)
        return fail(BN_EINVAL, "null device pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* d = p->ws.at<char>();
    const Meta m = meta_at(d, p->o, p->hm, &p->maps);
    Inputs in{d_v, d_g, d_t, d_t_nnz, d_seeds};
    const Scratch sc = scratch_at(d, p->o);
    Outputs out{d_ids, d_scores, d_n, d_failed, nullptr};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!p->prof.empty() && p->prof_n < p->prof.size() / 2) {
        e0 = p->prof[2 * p->prof_n];
        e1 = p->prof[2 * p->prof_n + 1];
        ++p->prof_n;
    }
    return enqueue_pipeline(p->h->e.ctx, p->h->e.c, p->z, m, in, sc, out, s, e0, e1);
}

int bn_plan_enqueue_scan(bn_plan* p, const uint64_t* d_v, uint64_t* d_r, void* stream) {
    if (!p || !d_v || !d_r) return fail(BN_EINVAL, "null argument");
    if (p->block) return fail(BN_EINVAL, "block plan: use bn_plan_enqueue_block");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* d = p->ws.at<char>();
    const RunLayout& o = p->o;
    CU(cudaMemsetAsync(d + o.err, 0, 4, s));
    launch_query_limbs(d_v, p->z.B, reinterpret_cast<QLimb*>(d + o.limbs), s);
    launch_scan(p->h->e.c.m_enc.at<uint64_t>(), reinterpret_cast<QLimb*>(d + o.limbs),
                reinterpret_cast<ScanSeg*>(d + o.segs), reinterpret_cast<uint64_t*>(d + o.seg_blk),
                (uint32_t)p->hm.segs.size(), p->hm.seg_blk.back(), d_r, p->h->e.ctx->num_sms,
                reinterpret_cast<uint32_t*>(d + o.err), s);
    CU(cudaGetLastError());
    return BN_OK;
}

int bn_plan_profile(bn_plan* p, uint32_t max_launches) {
    if (!p) return fail(BN_EINVAL, "null plan");
    if (p->block) return fail(BN_EINVAL, "block plans report their GEMM times through bn_plan_block_config");
    if (max_launches > 65536) return fail(BN_EINVAL, "max_launches = %u exceeds 65536", max_launches);
    for (cudaEvent_t e : p->prof) cudaEventDestroy(e);
    p->prof.assign(2ull * max_launches, nullptr);
    p->prof_n = 0;
    for (auto& e : p->prof) CU(cudaEventCreate(&e));
    return BN_OK;
}

int bn_plan_profile_read(bn_plan* p, float* ms, uint32_t cap, uint32_t* n) {
    if (!p || !n || (cap && !ms)) return fail(BN_EINVAL, "null argument");
    const uint32_t got = std::min(p->prof_n, cap);
    for (uint32_t i = 0; i < got; ++i) {
        CU(cudaEventSynchronize(p->prof[2 * i + 1]));
        CU(cudaEventElapsedTime(&ms[i], p->prof[2 * i], p->prof[2 * i + 1]));
    }
    *n = got;
    p->prof_n = 0;
    return BN_OK;
}

int bn_plan_status(bn_plan* p, uint32_t* device_flags) {
    if (!p || !device_flags) return fail(BN_EINVAL, "null argument");
    if (p->block) return block_plan_status(p->block, device_flags);
    uint32_t w[2] = {0, 0};
    CU(cudaMemcpy(&w[0], p->ws.at<char>() + p->o.err, 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&w[1], p->ws.at<char>() + p->o.flags, 4, cudaMemcpyDeviceToHost));
    *device_flags = w[0] | w[1];
    return BN_OK;
}

int bn_flat_block_prepare(bn_flat* f) {
    if (!f) return fail(BN_EINVAL, "null handle");
    if (!f->m) return fail(BN_EINVAL, "empty corpus");
    return block_prepare(f);
}

int bn_flat_block_plan(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k, uint32_t flags, bn_plan** out) {
    if (!f || !out) return fail(BN_EINVAL, "null argument");
    flags &= BN_BLOCK_AUTOTUNE;
    *out = nullptr;
    BlockPlan* b = nullptr;
    TRY(block_plan_create(f, B, trials, k, flags, &b));
    auto* p = new bn_plan();
    p->h = f;
    p->block = b;
    *out = p;
    return BN_OK;
}

int bn_plan_block_config(const bn_plan* p, uint32_t config[6], float tuned_ms[2]) {
    if (!p || !config) return fail(BN_EINVAL, "null argument");
    if (!p->block) return fail(BN_EINVAL, "not a block plan");
    block_plan_config(p->block, config, tuned_ms);
    return BN_OK;
}

int bn_plan_enqueue_block(bn_plan* p, const uint64_t* d_v, const uint64_t* d_g, const uint32_t* d_t,
                          const uint32_t* d_t_nnz, const uint8_t* d_block_seed, uint32_t* d_ids, int64_t* d_scores,
                          uint32_t* d_n, int32_t* d_failed, void* stream) {
    if (!p) return fail(BN_EINVAL, "null plan");
    if (!p->block) return fail(BN_EINVAL, "not a block plan: use bn_plan_enqueue");
    return block_enqueue(*p->block, d_v, d_g, d_t, d_t_nnz, d_block_seed, d_ids, d_scores, d_n, d_failed,
                         static_cast<cudaStream_t>(stream), false);
}

static int cached_block_plan(bn_flat* f, uint32_t B, uint32_t trials, uint32_t k, uint32_t flags, BlockPlan** out) {
    if (f->block_cache && f->cache_B == B && f->cache_trials == trials && f->cache_k == k && f->cache_flags == flags) {
        *out = f->block_cache;
        return BN_OK;
    }
    if (f->block_cache) {
        block_plan_free(f->block_cache);
        f->block_cache = nullptr;
    }
    TRY(block_plan_create(f, B, trials, k, flags, &f->block_cache));
    f->cache_flags = flags;
    f->cache_B = B;
    f->cache_trials = trials;
    f->cache_k = k;
    *out = f->block_cache;
    return BN_OK;
}

int bn_flat_query_block(bn_flat* f, uint32_t B, const uint64_t* v_enc, const uint64_t* g, const uint32_t* t_idx,
                        const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* block_seed, uint32_t trials,
                        uint32_t k, uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_trial,
                        uint64_t* mv_out) {
    if (!f) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (!v_enc || !g || !t_nnz || (trials && !block_seed)) return fail(BN_EINVAL, "null query input");
    TRY(validate_residues(v_enc, (uint64_t)B * N, "v_enc"));
    TRY(validate_residues(g, (uint64_t)B * f->e.c.n1, "g"));
    uint64_t t_total = 0;
    for (uint32_t q = 0; q < B; ++q) t_total += t_nnz[q];
    if (t_total && (!t_idx || !t_sign)) return fail(BN_EINVAL, "t_idx / t_sign are null");
    std::lock_guard<std::mutex> gd(f->block_mu);
    BlockPlan* b = nullptr;
    TRY(cached_block_plan(f, B, trials, k, 0, &b));
    return block_query_host(*b, v_enc, g, t_idx, t_sign, t_nnz, block_seed, ids, scores, n_hits, failed_trial, mv_out);
}

int bn_flat_verify_block(bn_flat* f, uint32_t B, const uint64_t* r, const uint64_t* v_enc, const uint8_t* block_seed,
                         uint32_t trials, int32_t* failed_trial, uint64_t* ur, uint64_t* zv) {
    if (!f || !r || !v_enc || !block_seed || !failed_trial) return fail(BN_EINVAL, "null argument");
    if (B == 0) return BN_OK;
    if (trials == 0) return fail(BN_EINVAL, "trials must be >= 1");
    TRY(validate_residues(v_enc, (uint64_t)B * N, "v_enc"));
    TRY(validate_residues(r, (uint64_t)B * f->m, "r"));
    std::lock_guard<std::mutex> gd(f->block_mu);
    BlockPlan* b = nullptr;
    TRY(cached_block_plan(f, B, trials, 0, BLOCK_VERIFY_ONLY, &b));
    return block_verify_host(*b, r, v_enc, block_seed, failed_trial, ur, zv);
}

int bn_plan_destroy(bn_plan* p) {
    delete p;
    return BN_OK;
}

// ---------------------------------------------------------------- IVF
static int check_offsets(uint32_t nlist, const uint64_t* off) {
    if (!off) return fail(BN_EINVAL, "null list_offsets");
    if (off[0] != 0) return fail(BN_EINVAL, "list_offsets[0] must be 0");
    for (uint32_t c = 0; c < nlist; ++c) {
        if (off[c + 1] < off[c]) return fail(BN_EINVAL, "list_offsets not monotone at %u", c);
        if (off[c + 1] - off[c] > 0xffffffffull) return fail(BN_EINVAL, "list %u larger than 2^32 rows", c);
    }
    return BN_OK;
}

// Internal hooks for bn_noalloc.cu (not part of the public header).
int bn_internal_set_error(int code, const char* msg) { return fail(code, "%s", msg); }

int bn_internal_flat_view(const bn_flat* f, int* device, const uint64_t** d_m_enc, uint64_t* rows, int* num_sms,
                          int* debug_draw_hit) {
    if (!f) return fail(BN_EINVAL, "null handle");
    *device = f->e.ctx->device;
    *debug_draw_hit = f->e.ctx->debug_draw_hit;
    *d_m_enc = f->e.c.m_enc.at<uint64_t>();
    *rows = f->m;
    *num_sms = f->e.ctx->num_sms;
    return BN_OK;
}

int bn_ivf_build(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, const uint32_t* ids, const uint64_t* m_enc,
                 const uint64_t* a_l, const uint64_t* h, uint32_t n, uint32_t n1, bn_ivf** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    TRY(check_offsets(nlist, off));
    const uint64_t rows = off[nlist];
    if (rows && (!ids || !m_enc || !a_l || !h)) return fail(BN_EINVAL, "null corpus array");
    TRY(validate_residues(m_enc, rows * N, "m_enc"));
    TRY(validate_residues(a_l, rows * n1, "a_l"));
    TRY(validate_residues(h, rows * n1, "h"));
    auto* v = new bn_ivf();
    int rc = engine_init(v->e, ctx);
    v->nlist = nlist;
    v->offsets.assign(off, off + nlist + 1);
    Corpus& c = v->e.c;
    c.rows = rows;
    c.n1 = n1;
    if (rc == BN_OK) rc = c.m_enc.alloc(ctx, rows * N * 8);
    if (rc == BN_OK && rows && cudaMemcpy(c.m_enc.p, m_enc, rows * N * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(BN_ECUDA, "upload m_enc failed");
    if (rc == BN_OK) rc = corpus_tmap(c);
    if (rc == BN_OK) rc = c.ids.alloc(ctx, std::max<uint64_t>(rows, 1) * 4);
    if (rc == BN_OK && rows && cudaMemcpy(c.ids.p, ids, rows * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(BN_ECUDA, "upload ids failed");
    if (rc == BN_OK) rc = upload_colmajor(ctx, a_l, rows, n1, c.al_cm, v->e.stream);
    if (rc == BN_OK) rc = upload_colmajor(ctx, h, rows, n1, c.h_cm, v->e.stream);
    if (rc != BN_OK) {
        engine_free(v->e);
        delete v;
        return rc;
    }
    *out = v;
    return BN_OK;
}

int bn_ivf_attach_client(bn_ivf* v, const uint64_t* L, const uint64_t* m_plain, bn_sparse_csr s_mat) {
    if (!v) return fail(BN_EINVAL, "null handle");
    std::lock_guard<std::mutex> g(v->e.mu);
    CU(cudaSetDevice(v->e.ctx->device));
    TRY(validate_residues(m_plain, v->e.c.rows * N, "m_plain"));
    return attach_client(v->e.ctx, v->e.c, L, m_plain, s_mat, v->e.stream);
}

int bn_ivf_build_from_plain(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, const uint32_t* ids, const uint64_t* m_q,
                            uint32_t n, uint32_t n1, const uint64_t* L, const uint64_t* H, bn_sparse_csr S,
                            bn_ivf** out) {
    if (!ctx || !out) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    TRY(check_offsets(nlist, off));
    const uint64_t rows = off[nlist];
    if (rows && !ids) return fail(BN_EINVAL, "null ids");
    TRY(check_plain_inputs(m_q, rows, L, H, n1, S));
    auto* v = new bn_ivf();
    int rc = engine_init(v->e, ctx);
    v->nlist = nlist;
    v->offsets.assign(off, off + nlist + 1);
    if (rc == BN_OK) rc = build_corpus_from_plain(ctx, v->e.c, m_q, rows, n1, L, H, S, v->e.stream);
    if (rc == BN_OK) rc = v->e.c.ids.alloc(ctx, std::max<uint64_t>(rows, 1) * 4);
    if (rc == BN_OK && rows && cudaMemcpy(v->e.c.ids.p, ids, rows * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(BN_ECUDA, "upload ids failed");
    if (rc != BN_OK) {
        engine_free(v->e);
        delete v;
        return rc;
    }
    *out = v;
    return BN_OK;
}

int bn_ivf_destroy(bn_ivf* v) {
    if (!v) return BN_OK;
    engine_free(v->e);
    delete v;
    return BN_OK;
}

int bn_ivf_info(const bn_ivf* v, uint64_t* rows, uint64_t* bytes) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (rows) *rows = v->e.c.rows;
    if (bytes) *bytes = v->e.c.bytes();
    return BN_OK;
}

int bn_ivf_compute_products(bn_ivf* v, uint32_t ci, const uint64_t* v_enc, uint64_t* r, uint64_t* m_out) {
    if (!v || !m_out) return fail(BN_EINVAL, "null argument");
    *m_out = 0;
    if (ci >= v->nlist) return BN_OK;
    const uint64_t row0 = v->offsets[ci], m = v->offsets[ci + 1] - row0;
    if (!m) return BN_OK;
    std::lock_guard<std::mutex> g(v->e.mu);
    TRY(run_scan(v->e, row0, m, v_enc, 1, r));
    *m_out = m;
    return BN_OK;
}

int bn_ivf_decode_dense_terms(bn_ivf* v, uint32_t ci, const uint64_t* g, const uint64_t* lt, uint64_t* out,
                              uint64_t* m_out) {
    if (!v || !m_out) return fail(BN_EINVAL, "null argument");
    *m_out = 0;
    if (ci >= v->nlist) return BN_OK;
    const uint64_t row0 = v->offsets[ci], m = v->offsets[ci + 1] - row0;
    if (!m) return BN_OK;
    std::lock_guard<std::mutex> gd(v->e.mu);
    // dense_terms_kernel walks columns with stride = its row count, so give
    // it a compact copy of this list's AL / H columns.
    Engine& e = v->e;
    const uint32_t n1 = e.c.n1;
    DevMem al, hh;
    TRY(al.alloc(e.ctx, m * n1 * 8));
    TRY(hh.alloc(e.ctx, m * n1 * 8));
    CU(cudaMemcpy2DAsync(al.p, m * 8, e.c.al_cm.at<uint64_t>() + row0, e.c.rows * 8, m * 8, n1, cudaMemcpyDeviceToDevice, e.stream));
    CU(cudaMemcpy2DAsync(hh.p, m * 8, e.c.h_cm.at<uint64_t>() + row0, e.c.rows * 8, m * 8, n1, cudaMemcpyDeviceToDevice, e.stream));
    TRY(validate_residues(g, n1, "g"));
    TRY(validate_residues(lt, n1, "lt_venc"));
    Layout L;
    const uint64_t o_g = L.take<uint64_t>(n1), o_x = L.take<uint64_t>(n1), in_end = L.off, o_o = L.take<uint64_t>(m);
    TRY(e.ws.reserve(e.ctx, L.off));
    TRY(e.host.reserve(in_end));
    char* h = e.host.at<char>();
    memcpy(h + o_g, g, n1 * 8ull);
    memcpy(h + o_x, lt, n1 * 8ull);
    char* d = e.ws.at<char>();
    CU(cudaMemcpyAsync(d, h, in_end, cudaMemcpyHostToDevice, e.stream));
    launch_dense_terms(al.at<uint64_t>(), hh.at<uint64_t>(), m, n1, reinterpret_cast<uint64_t*>(d + o_g),
                       reinterpret_cast<uint64_t*>(d + o_x), reinterpret_cast<uint64_t*>(d + o_o), e.stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, d + o_o, m * 8, cudaMemcpyDeviceToHost, e.stream));
    CU(cudaStreamSynchronize(e.stream));
    *m_out = m;
    return BN_OK;
}

int bn_ivf_verify(bn_ivf* v, uint32_t ci, const uint64_t* r, const uint64_t* v_enc, const uint8_t v_seed[32],
                  uint32_t trials, int32_t* failed_trial, uint64_t* ur, uint64_t* zv) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (ci >= v->nlist) return fail(BN_EINVAL, "list %u out of range", ci);
    std::lock_guard<std::mutex> g(v->e.mu);
    const uint64_t row0 = v->offsets[ci], m = v->offsets[ci + 1] - row0;
    return run_verify(v->e, row0, m, r, v_enc, v_seed, trials, failed_trial, ur, zv);
}

int bn_ivf_query(bn_ivf* v, uint32_t B, uint32_t nprobe, const uint32_t* probes, const uint64_t* v_enc, const uint64_t* g,
                 const uint32_t* t_idx, const int8_t* t_sign, const uint32_t* t_nnz, const uint8_t* v_seeds,
                 uint32_t trials, uint32_t k, uint32_t* ids, int64_t* scores, uint32_t* n_hits, int32_t* failed_cluster,
                 int32_t* failed_trial) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (nprobe && !probes) return fail(BN_EINVAL, "null probes");
    std::lock_guard<std::mutex> gd(v->e.mu);
    HostMeta hm;
    uint64_t out = 0;
    for (uint32_t b = 0; b < B; ++b) {
        const uint32_t seg0 = (uint32_t)hm.segs.size();
        for (uint32_t p = 0; p < nprobe; ++p) {
            const uint32_t ci = probes[(uint64_t)b * nprobe + p];
            if (ci >= v->nlist) return fail(BN_EINVAL, "probe %u of query %u names list %u of %u", p, b, ci, v->nlist);
            const uint64_t row0 = v->offsets[ci], m = v->offsets[ci + 1] - row0;
            if (!m) continue;  // ivf.rs:787-789 skips empty clusters
            hm.segs.push_back(ScanSeg{row0, out, (uint32_t)m, b});
            hm.vsegs.push_back(VerifySeg{row0, out, (uint32_t)m, b});
            hm.seg_cluster.push_back(ci);
            hm.max_rows = std::max(hm.max_rows, m);
            out += m;
        }
        hm.dq.push_back(DecodeQuery{seg0, (uint32_t)hm.segs.size() - seg0});
    }
    hm.total_out = out;
    finish_meta(hm);
    std::vector<int32_t> vf;
    TRY(run_query(v->e, hm, B, v_enc, g, t_idx, t_sign, t_nnz, v_seeds, trials, k, ids, scores, n_hits, vf, nullptr, nullptr));
    for (uint32_t b = 0; b < B; ++b) {
        int32_t fc = -1, ft = -1;
        const DecodeQuery& dq = hm.dq[b];
        for (uint32_t s = dq.seg0; s < dq.seg0 + dq.nseg; ++s)
            if (vf[s] >= 0) {
                fc = (int32_t)hm.seg_cluster[s];
                ft = vf[s];
                break;
            }
        if (failed_cluster) failed_cluster[b] = fc;
        if (failed_trial) failed_trial[b] = ft;
    }
    return BN_OK;
}

// ---------------------------------------------------------------- keygen
int bn_keygen_h_s(bn_ctx* ctx, const uint8_t* h_seed, uint64_t m, uint32_t n1, uint64_t* H, uint64_t* s_rowptr,
                  uint32_t* s_idx, int8_t* s_sign, uint64_t s_cap, uint64_t* nnz) {
    if (!ctx || !h_seed || !nnz || (m && (!H || !s_rowptr))) return fail(BN_EINVAL, "null argument");
    TRY(check_shape(N, n1));
    *nnz = 0;
    if (!m) {
        if (s_rowptr) s_rowptr[0] = 0;
        return BN_OK;
    }
    CU(cudaSetDevice(ctx->device));
    cudaStream_t s;
    CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int rc = BN_OK;
    {
        DevMem dH, rp, ix, sg;
        std::vector<uint64_t> hrp;
        const uint64_t off[2] = {0, m};
        rc = keygen_lists(ctx, 1, off, h_seed, n1, dH, rp, ix, sg, hrp, s);
        if (rc == BN_OK) {
            *nnz = hrp[m];
            if (hrp[m] > s_cap) {
                rc = fail(BN_EINVAL, "S has %llu entries, more than s_cap = %llu", (unsigned long long)hrp[m],
                          (unsigned long long)s_cap);
            } else {
                memcpy(s_rowptr, hrp.data(), (m + 1) * 8);
                cudaError_t e = cudaMemcpyAsync(H, dH.p, m * n1 * 8, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess && hrp[m]) e = cudaMemcpyAsync(s_idx, ix.p, hrp[m] * 4, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess && hrp[m]) e = cudaMemcpyAsync(s_sign, sg.p, hrp[m], cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) rc = fail(BN_ECUDA, "keygen copy-back: %s", cudaGetErrorString(e));
            }
        }
    }
    cudaStreamDestroy(s);
    return rc;
}

int bn_flat_build_keygen(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L,
                         const uint8_t* h_seed, bn_flat** out) {
    if (!ctx || !out || !h_seed || !L || (m && !m_q)) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    if (m > 0xffffffffull) return fail(BN_EINVAL, "cluster size must fit in u32");
    TRY(validate_residues(m_q, m * N, "m_q"));
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    auto* f = new bn_flat();
    int rc = engine_init(f->e, ctx);
    f->m = m;
    if (rc == BN_OK) {
        DevMem H, rp, ix, sg;
        std::vector<uint64_t> hrp;
        const uint64_t off[2] = {0, m};
        rc = keygen_lists(ctx, 1, off, h_seed, n1, H, rp, ix, sg, hrp, f->e.stream);
        if (rc == BN_OK) rc = build_corpus_device_keys(ctx, f->e.c, m_q, m, n1, L, H, hrp.data(), rp, ix, sg, f->e.stream);
    }
    if (rc != BN_OK) {
        engine_free(f->e);
        delete f;
        return rc;
    }
    *out = f;
    return BN_OK;
}

int bn_ivf_build_keygen(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, const uint32_t* ids, const uint64_t* m_q,
                        uint32_t n, uint32_t n1, const uint64_t* L, uint64_t upload_seed, bn_ivf** out) {
    return bn::api::ivf_build_keygen_from(ctx, nlist, off, ids, m_q, n, n1, L, upload_seed, 0, out);
}

}  // extern "C"

namespace bn {
namespace api {

int ivf_build_keygen_from(bn_ctx* ctx, uint32_t nlist, const uint64_t* off, const uint32_t* ids, const uint64_t* m_q,
                          uint32_t n, uint32_t n1, const uint64_t* L, uint64_t upload_seed, uint32_t list0,
                          bn_ivf** out) {
    if (!ctx || !out || !L) return fail(BN_EINVAL, "null argument");
    *out = nullptr;
    TRY(check_shape(n, n1));
    TRY(check_offsets(nlist, off));
    const uint64_t rows = off[nlist];
    if (rows && (!ids || !m_q)) return fail(BN_EINVAL, "null corpus array");
    TRY(validate_residues(m_q, rows * N, "m_q"));
    TRY(validate_residues(L, (uint64_t)N * n1, "l_subspace"));
    std::vector<uint8_t> seeds(32ull * std::max<uint32_t>(nlist, 1));
    for (uint32_t c = 0; c < nlist; ++c) derive_h_seed(upload_seed, list0 + c, &seeds[32ull * c]);  // ivf.rs:258-264
    auto* v = new bn_ivf();
    int rc = engine_init(v->e, ctx);
    v->nlist = nlist;
    v->offsets.assign(off, off + nlist + 1);
    if (rc == BN_OK) {
        DevMem H, rp, ix, sg;
        std::vector<uint64_t> hrp;
        rc = keygen_lists(ctx, nlist, off, seeds.data(), n1, H, rp, ix, sg, hrp, v->e.stream);
        if (rc == BN_OK) rc = build_corpus_device_keys(ctx, v->e.c, m_q, rows, n1, L, H, hrp.data(), rp, ix, sg, v->e.stream);
    }
    if (rc == BN_OK) rc = v->e.c.ids.alloc(ctx, std::max<uint64_t>(rows, 1) * 4);
    if (rc == BN_OK && rows && cudaMemcpy(v->e.c.ids.p, ids, rows * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(BN_ECUDA, "upload ids failed");
    if (rc != BN_OK) {
        engine_free(v->e);
        delete v;
        return rc;
    }
    *out = v;
    return BN_OK;
}

}  // namespace api
}  // namespace bn

extern "C" {

int bn_encrypt_cluster(bn_ctx* ctx, const uint64_t* m_q, uint64_t m, uint32_t n, uint32_t n1, const uint64_t* L,
                       const uint64_t* H, bn_sparse_csr S, uint64_t* m_enc, uint64_t* a_l) {
    if (!ctx) return fail(BN_EINVAL, "null ctx");
    TRY(check_shape(n, n1));
    TRY(check_plain_inputs(m_q, m, L, H, n1, S));
    if (m && (!m_enc || !a_l)) return fail(BN_EINVAL, "null output");
    if (!m) return BN_OK;
    CU(cudaSetDevice(ctx->device));
    cudaStream_t s;
    CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int rc = BN_OK;
    {
        DevMem d_mq, d_L, d_H, enc, al;
        rc = d_mq.alloc(ctx, m * N * 8);
        if (rc == BN_OK) rc = d_L.alloc(ctx, (uint64_t)N * n1 * 8);
        if (rc == BN_OK) rc = d_H.alloc(ctx, m * n1 * 8);
        if (rc == BN_OK) {
            cudaMemcpyAsync(d_mq.p, m_q, m * N * 8, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_L.p, L, (uint64_t)N * n1 * 8, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_H.p, H, m * n1 * 8, cudaMemcpyHostToDevice, s);
            rc = device_encrypt(ctx, d_mq.at<uint64_t>(), m, n1, d_L.at<uint64_t>(), d_H.at<uint64_t>(), S, enc, al, s);
        }
        if (rc == BN_OK) {
            cudaMemcpyAsync(m_enc, enc.p, m * N * 8, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(a_l, al.p, m * n1 * 8, cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = fail(BN_ECUDA, "encrypt: %s", cudaGetErrorString(e));
        }
    }
    cudaStreamDestroy(s);
    return rc;
}

}  // extern "C"
