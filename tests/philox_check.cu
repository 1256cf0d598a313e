// philox_check.cu -- compares include/hp_rng.h's Philox4x32-10 with curand's
// Philox4_32_10 generator on the device (test helper for tests/test_gpu_ops.py).
// curand_init(seed, subsequence, 0, &st) starts from counter
// (0, 0, subsequence_lo, subsequence_hi) and key (seed_lo, seed_hi); the
// first curand4() returns the block for that counter.
#include <cstdio>
#include <curand_kernel.h>
#include "hp_rng.h"

__global__ void k(int n, unsigned long long *seeds, unsigned long long *subs, uint4 *ref, uint4 *mine) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    curandStatePhilox4_32_10_t st;
    curand_init(seeds[t], subs[t], 0, &st);
    ref[t] = curand4(&st);
    hp_u4 c;
    c.x = 0; c.y = 0; c.z = (uint32_t)subs[t]; c.w = (uint32_t)(subs[t] >> 32);
    hp_u4 o = hp_philox4x32_10(c, (uint32_t)seeds[t], (uint32_t)(seeds[t] >> 32));
    mine[t] = make_uint4(o.x, o.y, o.z, o.w);
}

int main() {
    const int n = 4096;
    unsigned long long hs[n], hq[n];
    unsigned long long x = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < n; i++) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17; hs[i] = x;
        x ^= x << 13; x ^= x >> 7; x ^= x << 17; hq[i] = (i < 8) ? (unsigned long long)i : x;
    }
    unsigned long long *ds, *dq;
    uint4 *dr, *dm;
    cudaMalloc(&ds, sizeof hs); cudaMalloc(&dq, sizeof hq);
    cudaMalloc(&dr, n * sizeof(uint4)); cudaMalloc(&dm, n * sizeof(uint4));
    cudaMemcpy(ds, hs, sizeof hs, cudaMemcpyHostToDevice);
    cudaMemcpy(dq, hq, sizeof hq, cudaMemcpyHostToDevice);
    k<<<(n + 255) / 256, 256>>>(n, ds, dq, dr, dm);
    static uint4 r[n], m[n];
    cudaMemcpy(r, dr, sizeof r, cudaMemcpyDeviceToHost);
    cudaMemcpy(m, dm, sizeof m, cudaMemcpyDeviceToHost);
    int bad = 0;
    for (int i = 0; i < n; i++)
        if (r[i].x != m[i].x || r[i].y != m[i].y || r[i].z != m[i].z || r[i].w != m[i].w) {
            if (bad < 4) printf("i=%d curand %08x %08x %08x %08x mine %08x %08x %08x %08x\n", i, r[i].x, r[i].y, r[i].z, r[i].w, m[i].x, m[i].y, m[i].z, m[i].w);
            bad++;
        }
    // the host build of the same header agrees with the device build
    int hostbad = 0;
    for (int i = 0; i < n; i++) {
        hp_u4 c; c.x = 0; c.y = 0; c.z = (uint32_t)hq[i]; c.w = (uint32_t)(hq[i] >> 32);
        hp_u4 o = hp_philox4x32_10(c, (uint32_t)hs[i], (uint32_t)(hs[i] >> 32));
        if (o.x != m[i].x || o.y != m[i].y || o.z != m[i].z || o.w != m[i].w) hostbad++;
    }
    printf("checked %d mismatches %d host-vs-device %d\n", n, bad, hostbad);
    return (bad || hostbad) ? 1 : 0;
}
