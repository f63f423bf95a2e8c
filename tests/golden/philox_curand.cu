// Golden-vector generator: cuRAND's Philox4_32_10 (a third-party
// implementation of Philox4x32-10), called on the GPU for a set of
// (seed, subsequence, offset) triples.  Prints JSON on stdout.
// Built and run by gen_philox_curand.py.
#include <cstdio>
#include <cstdint>
#include <curand_kernel.h>

struct Case {
    unsigned long long seed, subseq, offset;
};

__global__ void gen(const Case* cs, uint4* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandStatePhilox4_32_10_t st;
    curand_init(cs[i].seed, cs[i].subseq, cs[i].offset, &st);
    out[i] = curand4(&st);
}

int main() {
    const int n = 96;
    Case h[n];
    unsigned long long x = 0x243F6A8885A308D3ull;
    auto next = [&]() {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        return x;
    };
    for (int i = 0; i < n; ++i) {
        h[i].seed = (i < 4) ? (unsigned long long)i : next();
        h[i].subseq = (i % 3 == 0) ? 0ull : next() >> (i % 40);
        h[i].offset = ((i % 2) ? next() >> (i % 30) : (unsigned long long)i) * 4ull;  // multiple of 4
    }
    Case* d = nullptr;
    uint4* o = nullptr;
    cudaMalloc(&d, sizeof(h));
    cudaMalloc(&o, n * sizeof(uint4));
    cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    gen<<<1, 128>>>(d, o, n);
    uint4 r[n];
    if (cudaMemcpy(r, o, sizeof(r), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    printf("{\"generator\": \"curandStatePhilox4_32_10_t via curand_init(seed, subsequence, offset) + curand4\",\n");
    printf(" \"cases\": [\n");
    for (int i = 0; i < n; ++i)
        printf("  {\"seed\": %llu, \"subsequence\": %llu, \"offset\": %llu, \"out\": [%u, %u, %u, %u]}%s\n", h[i].seed,
               h[i].subseq, h[i].offset, r[i].x, r[i].y, r[i].z, r[i].w, i + 1 < n ? "," : "");
    printf(" ]}\n");
    cudaFree(d);
    cudaFree(o);
    return 0;
}
