"""Generate tests/golden/cxx_symbols.txt: the mangled names of the reference's
C++ API for the MSM path, as a translation unit compiled against the
reference's own headers (include/curve.h, include/fp_kernels.h,
include/fp2_kernels.h) references them.  Run where the reference sources are
available:

    python tests/golden/make_cxx_symbols.py /path/to/gpu_msm

The fixture lets the CPU tests check that libgpu_msm_b200.so exports every
one of these symbols without the reference being present.
"""
import os
import subprocess
import sys
import tempfile

TU = r'''
#include "curve.h"
#include "fp_kernels.h"
#include "fp2_kernels.h"
void* refs[] = {
  (void*)&init_device_generators,
  (void*)&point_msm_u64_async_g1, (void*)&point_msm_u64_g1,
  (void*)&point_msm_u64_async_g2, (void*)&point_msm_u64_g2,
  (void*)&point_msm_async<G1Point>, (void*)&point_msm<G1Point>,
  (void*)&point_msm_async<G2Point>, (void*)&point_msm<G2Point>,
  (void*)&point_to_montgomery_batch_async<G1Point>, (void*)&point_to_montgomery_batch<G1Point>,
  (void*)&point_to_montgomery_batch_async<G2Point>, (void*)&point_to_montgomery_batch<G2Point>,
  (void*)&point_at_infinity_async<G1Point>, (void*)&point_at_infinity<G1Point>,
  (void*)&point_at_infinity_async<G2Point>, (void*)&point_at_infinity<G2Point>,
  (void*)&fp_add_array_host, (void*)&fp_mul_array_host,
  (void*)&fp_add_array_device, (void*)&fp_mul_array_device,
  (void*)&fp2_add_array_host, (void*)&fp2_mul_array_host,
};
// overloaded names (the stream APIs share them with the __host__ __device__
// element functions): referenced by calls whose argument types pick the
// stream forms; never run
template <class P>
void point_calls(cudaStream_t s, uint32_t g, P *p, const uint64_t *k) {
  point_add_async<P>(s, g, p, p, p); point_add<P>(s, g, p, p, p);
  point_double_async<P>(s, g, p, p); point_double<P>(s, g, p, p);
  point_neg_async<P>(s, g, p, p); point_neg<P>(s, g, p, p);
  point_scalar_mul_u64_async<P>(s, g, p, p, 3); point_scalar_mul_u64<P>(s, g, p, p, 3);
  point_scalar_mul_async<P>(s, g, p, p, k, 5); point_scalar_mul<P>(s, g, p, p, k, 5);
  point_to_montgomery_async<P>(s, g, p, p); point_to_montgomery<P>(s, g, p, p);
  point_from_montgomery_async<P>(s, g, p, p); point_from_montgomery<P>(s, g, p, p);
}
void element_calls(cudaStream_t s, uint32_t g, Fp *f, Fp2 *e, G1Point *p1, G2Point *p2, const uint64_t *k) {
  fp_add_async(s, g, f, f, f); fp_add(s, g, f, f, f);
  fp_sub_async(s, g, f, f, f); fp_sub(s, g, f, f, f);
  fp_mul_async(s, g, f, f, f); fp_mul(s, g, f, f, f);
  fp_neg_async(s, g, f, f); fp_neg(s, g, f, f);
  fp_inv_async(s, g, f, f); fp_inv(s, g, f, f);
  fp_div_async(s, g, f, f, f); fp_div(s, g, f, f, f);
  fp_copy_async(s, g, f, f); fp_copy(s, g, f, f);
  fp_zero_async(s, g, f); fp_zero(s, g, f);
  fp_one_async(s, g, f); fp_one(s, g, f);
  fp_to_montgomery_async(s, g, f, f); fp_to_montgomery(s, g, f, f);
  fp_from_montgomery_async(s, g, f, f); fp_from_montgomery(s, g, f, f);
  fp_mont_mul_async(s, g, f, f, f); fp_mont_mul(s, g, f, f, f);
  fp2_add_async(s, g, e, e, e); fp2_add(s, g, e, e, e);
  fp2_sub_async(s, g, e, e, e); fp2_sub(s, g, e, e, e);
  fp2_mul_async(s, g, e, e, e); fp2_mul(s, g, e, e, e);
  fp2_square_async(s, g, e, e); fp2_square(s, g, e, e);
  fp2_neg_async(s, g, e, e); fp2_neg(s, g, e, e);
  fp2_conjugate_async(s, g, e, e); fp2_conjugate(s, g, e, e);
  fp2_inv_async(s, g, e, e); fp2_inv(s, g, e, e);
  fp2_div_async(s, g, e, e, e); fp2_div(s, g, e, e, e);
  fp2_copy_async(s, g, e, e); fp2_copy(s, g, e, e);
  point_calls<G1Point>(s, g, p1, k);
  point_calls<G2Point>(s, g, p2, k);
  fp_add_gpu(s, g, f, f, f); fp_sub_gpu(s, g, f, f, f); fp_mul_gpu(s, g, f, f, f);
  fp_neg_gpu(s, g, f, f); fp_inv_gpu(s, g, f, f); fp_div_gpu(s, g, f, f, f);
  (void)fp_cmp_gpu(s, g, f, f); (void)fp_is_zero_gpu(s, g, f); (void)fp_is_one_gpu(s, g, f);
  fp_to_montgomery_gpu(s, g, f, f); fp_from_montgomery_gpu(s, g, f, f); fp_mont_mul_gpu(s, g, f, f, f);
  fp_copy_gpu(s, g, f, f); fp_cmov_gpu(s, g, f, f, 1); (void)fp_sqrt_gpu(s, g, f, f);
  (void)fp_is_quadratic_residue_gpu(s, g, f); fp_pow_u64_gpu(s, g, f, f, 3);
  fp2_add_gpu(e, e, e); fp2_sub_gpu(e, e, e); fp2_mul_gpu(e, e, e); fp2_neg_gpu(e, e);
  fp2_conjugate_gpu(e, e); fp2_square_gpu(e, e); fp2_inv_gpu(e, e); fp2_div_gpu(e, e, e);
  fp2_mul_by_i_gpu(e, e); fp2_frobenius_gpu(e, e); (void)fp2_cmp_gpu(e, e);
  (void)fp2_is_zero_gpu(e); (void)fp2_is_one_gpu(e); fp2_copy_gpu(e, e); fp2_cmov_gpu(e, e, 1);
}
'''


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_cxx_symbols.py <reference checkout>")
    ref = sys.argv[1]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cxx_symbols.txt")
    with tempfile.TemporaryDirectory() as d:
        src, obj = os.path.join(d, "refs.cu"), os.path.join(d, "refs.o")
        open(src, "w").write(TU)
        subprocess.check_call(["nvcc", "-std=c++17", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a", "-c", "-w", "-I", os.path.join(ref, "include"), "-o", obj, src])
        nm = subprocess.check_output(["nm", "-u", obj], text=True)
    syms = sorted(set(line.split()[-1] for line in nm.splitlines()
                      if any(k in line for k in ("point_", "fp_", "fp2_", "init_device_generators"))))
    with open(out, "w") as f:
        f.write("# mangled C++ symbols of the reference's MSM-path API (make_cxx_symbols.py)\n")
        for s in syms:
            f.write(s + "\n")
    print(f"wrote {len(syms)} symbols to {out}")


if __name__ == "__main__":
    main()
