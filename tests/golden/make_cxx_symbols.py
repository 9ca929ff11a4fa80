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
'''


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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
