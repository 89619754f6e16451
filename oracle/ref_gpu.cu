// ref_gpu.cu -- TEST AND MEASUREMENT INFRASTRUCTURE ONLY, never linked into
// the product.  Compiles the reference's own GPU scan kernel,
// bntm_compute_products (scorer-bntm/src/gpu/kernels.cu:100-178), from the
// reference source file where it lies (its path arrives as BNREF_KERNELS_CU
// from oracle/Makefile, target `ref`) for sm_100a, and exposes one C entry
// point that launches it with the reference's own launch shape
// (gpu/mod.rs:362-379: one 256-thread CTA per row), so that bench.py can time
// the reference kernel on the same B200 and corpus as the product's kernels
// and the tests can check its r against the oracle.
#include BNREF_KERNELS_CU

extern "C" int bnref_compute_products(const uint64_t* d_m_enc, const uint64_t* d_v_enc, uint64_t* d_r, uint32_t m,
                                      void* stream) {
    if (m == 0) return 0;
    bntm_compute_products<<<m, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_m_enc, d_v_enc, d_r, m);
    return static_cast<int>(cudaGetLastError());
}
