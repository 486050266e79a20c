"""The velocity kernel's face-density division (div_face_rcp in
csrc/pe_kernels_pair.cuh) against IEEE float32 division, bit for bit, on the
device: every numerator class (zeros, subnormals, normals of all exponents,
infinities) and the densities of the disks (couplant 300, ice 917, their
face average 608.5) plus random positive divisors. Includes the exact
subnormal midpoints a / 300 = (2M + 1) 2^-150, where a product with a
rounded reciprocal would round the wrong way. The probe is compiled here
against the library's own header (nvcc, same flags as the library)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200", "pefdtd", "csrc")

PROBE = r'''
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include "pe_kernels_pair.cuh"

__device__ unsigned int mix(unsigned long long x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return (unsigned int)x;
}

// numerator i of a sweep: random bit patterns (NaN excluded), small
// multiples of 2^-149, and odd multiples of 75 * 2^-148 (exact midpoints
// of a / 300)
__device__ float numerator(unsigned long long i)
{
    const unsigned int k = (unsigned int)(i % 4);
    const unsigned int h = mix(i);
    if (k == 0) {
        unsigned int u = h;
        if ((u & 0x7f800000u) == 0x7f800000u) u &= ~0x00400000u, u &= 0xff800000u;   // +-inf only
        float f; memcpy(&f, &u, 4); return f;
    }
    if (k == 1) { const unsigned int u = h & 0x00ffffffu; float f; memcpy(&f, &u, 4); return (h >> 31) ? -f : f; }
    if (k == 2) { const unsigned int u = (h & 0x0fffffffu) | 0x00800000u; float f; memcpy(&f, &u, 4); return f; }
    const unsigned int m = (h & 0x7fffu) * 2u + 1u;   // odd, 75 m < 2^24
    return ldexpf((float)(75u * m), -148);
}

__global__ void k_probe(float b, float yb, unsigned long long n, unsigned long long *bad,
                        unsigned int *first)
{
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const float a = numerator(i);
        const float want = a / b;
        const float own = pe::div_face_rcp(a, b, true, yb);
        const float other = pe::div_face_rcp(a, b, false, 0.0f);
        unsigned int w, g1, g2;
        memcpy(&w, &want, 4); memcpy(&g1, &own, 4); memcpy(&g2, &other, 4);
        if (w != g1 || w != g2) {
            if (atomicAdd(bad, 1ULL) == 0) { unsigned int ua; memcpy(&ua, &a, 4); first[0] = ua; first[1] = w; first[2] = g1; first[3] = g2; }
        }
    }
}

int main(int argc, char **argv)
{
    const unsigned long long n = 1ULL << 28;
    unsigned long long *bad; unsigned int *first;
    cudaMalloc(&bad, 8); cudaMalloc(&first, 16);
    int rc = 0;
    for (int k = 1; k < argc; ++k) {
        const float b = strtof(argv[k], nullptr);
        const float yb = 1.0f / b;
        cudaMemset(bad, 0, 8); cudaMemset(first, 0, 16);
        k_probe<<<1184, 256>>>(b, yb, n, bad, first);
        unsigned long long h = 0; unsigned int f[4] = {0, 0, 0, 0};
        cudaMemcpy(&h, bad, 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(f, first, 16, cudaMemcpyDeviceToHost);
        const cudaError_t e = cudaGetLastError();
        printf("b=%.9g n=%llu mismatches=%llu first a=%08x want=%08x own=%08x div=%08x err=%d\n", b, n, h,
               f[0], f[1], f[2], f[3], (int)e);
        if (h || e != cudaSuccess) rc = 1;
    }
    return rc;
}
'''


def test_face_division_bit_exact_against_ieee_float32():
    rng = np.random.default_rng(3)
    # densities of the disks, a power of two, an all-ones significand
    divisors = ["300", "917", "608.5", "1000", "1", "512",
                repr(float(np.frombuffer(np.uint32(0x447FFFFF).tobytes(), np.float32)[0]))] + \
               [repr(float(np.float32(v))) for v in
                                                      rng.uniform(50.0, 5000.0, 6)]
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.cu")
        exe = os.path.join(d, "probe")
        with open(src, "w") as f:
            f.write(PROBE)
        nvcc = os.environ.get("NVCC", "nvcc")
        subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-fmad=false",
                               "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", exe, src])
        r = subprocess.run([exe] + divisors, capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("mismatches=0 ") == len(divisors)
