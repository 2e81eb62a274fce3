// Checks the fast forms of sci_math.cuh against the full forms: every float bit pattern, and a
// sample of doubles (hashed 64-bit patterns and values spread over each function's ordinary
// range), through apply_lanes with and without `fast`. Prints one line per code and precision:
// "<name> <precision> <checked> <mismatches> <first mismatching input bits>". Test infrastructure:
// compiled and run by tests/test_fast_forms_gpu.py.
#include "chunk_kernel.cuh"

#include <cstdio>

using namespace sci_cuda;

__device__ unsigned long long mismatches[2][16];
__device__ unsigned long long first_bad[2][16];

__device__ __forceinline__ unsigned long long mix(unsigned long long v) {
    // splitmix64 finaliser
    v += 0x9e3779b97f4a7c15ull;
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}

template <typename T> __device__ __forceinline__ T element(unsigned long long index);
template <> __device__ __forceinline__ float element<float>(unsigned long long index) {
    return __uint_as_float(static_cast<unsigned>(index));
}
template <> __device__ __forceinline__ double element<double>(unsigned long long index) {
    const unsigned long long h = mix(index);
    switch (index & 3) {
    case 0: return __longlong_as_double(static_cast<long long>(h));                      // any pattern
    case 1: return (static_cast<double>(h >> 11) * 0x1p-53 - 0.5) * 1500.0;               // exp's range
    case 2: return static_cast<double>(h >> 11) * 0x1p-53 * 1e6;                          // log, positive
    default: return (static_cast<double>(h >> 11) * 0x1p-53 - 0.5) * 2.2e6;               // sin / cos reach
    }
}

template <int code, int slot, typename T>
__global__ void compare(unsigned long long start) {
    constexpr int N = Lanes<T>::count;
    const unsigned long long base =
        start + (static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x) * N;
    T a[N], b[N] = {}, c[N] = {}, full[N], fast[N];
    bool tail[N] = {};
#pragma unroll
    for (int e = 0; e < N; ++e) a[e] = element<T>(base + e);
    apply_lanes<code, false>(a, b, c, full, tail);
    apply_lanes<code, true>(a, b, c, fast, tail);
    unsigned bad = 0;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        if (bits(full[e]) != bits(fast[e])) {
            ++bad;
            atomicMin(&first_bad[sizeof(T) == 8][slot], static_cast<unsigned long long>(bits(a[e])));
        }
    }
    if (bad) atomicAdd(&mismatches[sizeof(T) == 8][slot], bad);
}

template <int code, int slot, typename T> bool sweep(const char *name, unsigned long long total) {
    constexpr unsigned threads = 256;
    const unsigned long long per = 1ull << 28;
    for (unsigned long long start = 0; start < total; start += per)
        compare<code, slot, T><<<static_cast<unsigned>(per / Lanes<T>::count / threads), threads>>>(start);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        std::printf("error %s\n", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    unsigned long long m[2][16], f[2][16];
    cudaMemcpyFromSymbol(m, mismatches, sizeof(m));
    cudaMemcpyFromSymbol(f, first_bad, sizeof(f));
    const int p = sizeof(T) == 8;
    std::printf("%s %s %llu %llu 0x%llx\n", name, p ? "double" : "float", total, m[p][slot], f[p][slot]);
    return true;
}

template <typename T> bool all(unsigned long long total) {
    return sweep<kExponential, 0, T>("exponential", total) && sweep<kLogarithm, 1, T>("logarithm", total) &&
           sweep<kSin, 2, T>("sin", total) && sweep<kCos, 3, T>("cos", total) && sweep<kTan, 4, T>("tan", total) &&
           sweep<kCsc, 5, T>("csc", total) && sweep<kSec, 6, T>("sec", total) && sweep<kCot, 7, T>("cot", total) &&
           sweep<kTanh, 8, T>("tanh", total) && sweep<kCoth, 9, T>("coth", total);
}

int main() {
    unsigned long long none[2][16];
    for (auto &row : none)
        for (auto &v : row) v = ~0ull;
    cudaMemcpyToSymbol(first_bad, none, sizeof(none));
    if (!all<float>(1ull << 32)) return 1;
    if (!all<double>(1ull << 31)) return 1;
    return 0;
}
