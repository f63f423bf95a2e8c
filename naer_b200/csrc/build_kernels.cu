// Device connectivity builders.  The reference builds its segmented CSR with
// count_connections / integrate_connections / generate_connections
// (include/naer/kernels/network.cl:14-107, driven by src/Network.cpp:421-569);
// its scan runs on a single work-item and its fill order depends on local
// atomics.  Here counts, a device scan (CUB, on the host side) and the fill
// are all parallel and the row order is fixed.
#include "build_kernels.cuh"

namespace naer {

__global__ void k_fill_u32(uint32_t* a, uint64_t n, uint32_t v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

// REF_BERNOULLI: source s (local index) is connected to target d (local
// index) iff uniform_rand(seed, d) < p, evaluated by the reference's
// work-item s*32 + d%32 (count_connections, network.cl:25-41; the launch is
// src_size*32 items in groups of 32, Network.cpp:462).
__device__ __forceinline__ void bern_draw(const ConnBuild& cb, uint32_t s, uint32_t d, bool& conn,
                                          double& x, uint32_t& word0) {
    const u32x4 r = philox4x32_10(d, 0u, 0u, 0u, s * 32u + (d & 31u), cb.seed_lo);
    x = (double)r.v[2] / 4294967295.0;
    conn = x < cb.p;
    word0 = r.v[0];
}

__global__ void k_bern_count(ConnBuild cb, uint32_t* cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < cb.src_size; s += nw) {
        uint32_t c = 0;
        for (uint32_t d0 = 0; d0 < cb.dst_size; d0 += 32) {
            const uint32_t d = d0 + lane;
            bool conn = false;
            double x;
            uint32_t w0;
            if (d < cb.dst_size) bern_draw(cb, s, d, conn, x, w0);
            c += __popc(__ballot_sync(0xFFFFFFFFu, conn));
        }
        if (lane == 0) cnt[s] = c;
    }
}

__global__ void k_bern_fill(ConnBuild cb, const uint64_t* cursor, uint32_t* tgt, float* w,
                            uint8_t* dly) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < cb.src_size; s += nw) {
        uint64_t pos = cursor[cb.src_storage + s];
        for (uint32_t d0 = 0; d0 < cb.dst_size; d0 += 32) {
            const uint32_t d = d0 + lane;
            bool conn = false;
            double x = 0.0;
            uint32_t w0 = 0;
            if (d < cb.dst_size) bern_draw(cb, s, d, conn, x, w0);
            const uint32_t b = __ballot_sync(0xFFFFFFFFu, conn);
            if (conn) {
                const uint64_t o = pos + __popc(b & lt);
                tgt[o] = cb.dst_storage + d;
                w[o] = cb.weight == 0.0f ? conn_uniform_weight(cb.wmin, cb.wmax, __double2float_rn(x))
                                         : cb.weight;
                dly[o] = (uint8_t)conn_delay(cb.dmin, cb.dmax, w0);
            }
            pos += __popc(b);
        }
    }
}

// FIXED_OUTDEGREE: draw k of source s picks target umulhi(word, dst_size)
// from Philox(ctr {s, k/4, 0, 0}, key {seed_lo, seed_hi}) word k%4; the
// delay uses ctr word 2 = 1 and the random weight ctr word 2 = 2.
__global__ void k_outdeg_fill(ConnBuild cb, const uint64_t* cursor, uint32_t* tgt, float* w,
                              uint8_t* dly) {
    const uint32_t blocks = (cb.K + 3u) >> 2;
    const uint64_t total = (uint64_t)cb.src_size * blocks;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < total;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = (uint32_t)(it / blocks);
        const uint32_t b = (uint32_t)(it % blocks);
        const u32x4 rt = philox4x32_10(s, b, 0u, 0u, cb.seed_lo, cb.seed_hi);
        const u32x4 rd = philox4x32_10(s, b, 1u, 0u, cb.seed_lo, cb.seed_hi);
        u32x4 rw;
        if (cb.weight == 0.0f) rw = philox4x32_10(s, b, 2u, 0u, cb.seed_lo, cb.seed_hi);
        const uint64_t base = cursor[cb.src_storage + s];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t k = b * 4u + j;
            if (k >= cb.K) break;
            const uint64_t o = base + k;
            tgt[o] = cb.dst_storage + conn_pick(rt.v[j], cb.dst_size);
            w[o] = cb.weight == 0.0f ? conn_uniform_weight(cb.wmin, cb.wmax, conn_unit_float(rw.v[j]))
                                     : cb.weight;
            dly[o] = (uint8_t)conn_delay(cb.dmin, cb.dmax, rd.v[j]);
        }
    }
}

// FIXED_INDEGREE: draw k of target i picks source umulhi(word, src_size)
// from Philox(ctr {i, k/4, 0, 0}, key {seed_lo, seed_hi}) word k%4; delays
// and random weights as for FIXED_OUTDEGREE, indexed by (i, k).
__global__ void k_indeg_count(ConnBuild cb, uint32_t* cnt) {
    const uint32_t blocks = (cb.K + 3u) >> 2;
    const uint64_t total = (uint64_t)cb.dst_size * blocks;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < total;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(it / blocks);
        const uint32_t b = (uint32_t)(it % blocks);
        const u32x4 r = philox4x32_10(i, b, 0u, 0u, cb.seed_lo, cb.seed_hi);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (b * 4u + j >= cb.K) break;
            atomicAdd(cnt + conn_pick(r.v[j], cb.src_size), 1u);
        }
    }
}

// Fixed in-degree rows in canonical order without atomics: every draw
// d = target * K + k gets its source as a sort key and d as the value; a
// stable radix sort by source then lists each source's draws in ascending
// (target, k), the order the rows keep.
__global__ void k_indeg_keys(ConnBuild cb, uint32_t* keys, uint32_t* vals) {
    const uint32_t blocks = (cb.K + 3u) >> 2;
    const uint64_t total = (uint64_t)cb.dst_size * blocks;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < total;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(it / blocks);
        const uint32_t b = (uint32_t)(it % blocks);
        const u32x4 r = philox4x32_10(i, b, 0u, 0u, cb.seed_lo, cb.seed_hi);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t k = b * 4u + j;
            if (k >= cb.K) break;
            const uint32_t d = i * cb.K + k;
            keys[d] = conn_pick(r.v[j], cb.src_size);
            vals[d] = d;
        }
    }
}

// Sorted draw e (source s = keys[e], draw d = vals[e]) into its row: entry
// e - conn_off[s] of the connection's part of row s.
__global__ void k_indeg_finalize(ConnBuild cb, const uint32_t* keys, const uint32_t* vals, uint64_t total,
                                 const uint64_t* conn_off, const uint64_t* cursor, uint32_t* tgt,
                                 float* w, uint8_t* dly) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = keys[e];
        const uint32_t d = vals[e];
        const uint32_t i = d / cb.K;
        const uint32_t k = d - i * cb.K;
        const uint32_t b = k >> 2, j = k & 3u;
        const uint64_t o = cursor[cb.src_storage + s] + (e - conn_off[s]);
        tgt[o] = cb.dst_storage + i;
        const u32x4 rd = philox4x32_10(i, b, 1u, 0u, cb.seed_lo, cb.seed_hi);
        dly[o] = (uint8_t)conn_delay(cb.dmin, cb.dmax, rd.v[j]);
        if (cb.weight == 0.0f) {
            const u32x4 rw = philox4x32_10(i, b, 2u, 0u, cb.seed_lo, cb.seed_hi);
            w[o] = conn_uniform_weight(cb.wmin, cb.wmax, conn_unit_float(rw.v[j]));
        } else {
            w[o] = cb.weight;
        }
    }
}

__global__ void k_row_len_add(const uint32_t* cnt, uint32_t src_size, uint32_t src_storage,
                              uint64_t* len) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < src_size; s += gridDim.x * blockDim.x)
        len[src_storage + s] += cnt[s];
}

__global__ void k_row_pad(const uint64_t* len, uint32_t n, uint64_t* padded) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
        padded[i] = i < n ? (len[i] + (kRowAlign - 1)) / kRowAlign * kRowAlign : 0ull;
}

// Explicit connectivity: one warp per source row copies its synapses, in
// the given order, to the row's cursor (targets shifted to storage indices).
__global__ void k_explicit_fill(ConnBuild cb, const uint64_t* rp, const uint32_t* tg, const float* wv,
                                const uint8_t* dv, const uint64_t* cursor, uint32_t* tgt, float* w, uint8_t* dly) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < cb.src_size; s += nw) {
        const uint64_t b = rp[s], e = rp[s + 1], o = cursor[cb.src_storage + s];
        for (uint64_t j = b + lane; j < e; j += 32) {
            tgt[o + (j - b)] = cb.dst_storage + tg[j];
            w[o + (j - b)] = wv[j];
            dly[o + (j - b)] = dv[j];
        }
    }
}

__global__ void k_cursor_advance(const uint32_t* cnt, uint32_t src_size, uint32_t src_storage,
                                 uint64_t* cursor) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < src_size; s += gridDim.x * blockDim.x)
        cursor[src_storage + s] += cnt[s];
}

__global__ void k_pad_fill(const uint64_t* row_ptr, const uint64_t* len, uint32_t n, uint32_t* tgt,
                           float* w, uint8_t* dly) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (uint64_t o = row_ptr[i] + len[i]; o < row_ptr[i + 1]; ++o) {
            tgt[o] = kTgtSentinel;
            w[o] = 0.0f;
            dly[o] = 1;
        }
    }
}

// Delay-1 synapses of each row (valid entries only).
__global__ void k_count_d1(const uint64_t* row_ptr, const uint64_t* len, uint32_t n, const uint8_t* dly,
                           uint32_t* n1) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const uint64_t b = row_ptr[i], e = b + len[i];
        uint32_t c = 0;
        for (uint64_t j = b + lane; j < e; j += 32) c += dly[j] == 1 ? 1u : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (lane == 0) n1[i] = c;
    }
}

__global__ void k_row_pad_split(const uint64_t* len, const uint32_t* n1, uint32_t n, uint64_t* padded) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            padded[i] = 0;
            continue;
        }
        const uint64_t a = n1[i], b = len[i] - n1[i];
        padded[i] = (a + kRowAlign - 1) / kRowAlign * kRowAlign + (b + kRowAlign - 1) / kRowAlign * kRowAlign;
    }
}

// Stable partition of row i into [delay-1 part | pad | other part | pad]:
// one warp per row, ballots give every entry its place in its part.
__global__ void k_partition_d1(const uint64_t* row_ptr, const uint64_t* len, const uint32_t* n1, uint32_t n,
                               const uint64_t* row_ptr2, const uint32_t* tgt, const float* w, const uint8_t* dly,
                               uint32_t* tgt2, float* w2, uint8_t* dly2, uint32_t* row_mid) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const uint64_t b = row_ptr[i], L = len[i];
        const uint64_t o = row_ptr2[i], o_end = row_ptr2[i + 1];
        const uint32_t a = n1[i];
        const uint64_t mid = (a + kRowAlign - 1) / kRowAlign * kRowAlign;
        uint64_t r1 = 0, r2 = 0;
        for (uint64_t j0 = 0; j0 < L; j0 += 32) {
            const uint64_t j = j0 + lane;
            const bool valid = j < L;
            const bool one = valid && dly[b + j] == 1;
            const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, one);
            const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, valid && !one);
            if (valid) {
                const uint64_t q = one ? o + r1 + __popc(m1 & lt) : o + mid + r2 + __popc(m2 & lt);
                tgt2[q] = tgt[b + j];
                w2[q] = w[b + j];
                dly2[q] = dly[b + j];
            }
            r1 += __popc(m1);
            r2 += __popc(m2);
        }
        for (uint64_t q = o + a + lane; q < o + mid; q += 32) {
            tgt2[q] = kTgtSentinel;
            w2[q] = 0.0f;
            dly2[q] = 1;
        }
        for (uint64_t q = o + mid + (L - a) + lane; q < o_end; q += 32) {
            tgt2[q] = kTgtSentinel;
            w2[q] = 0.0f;
            dly2[q] = 1;
        }
        if (lane == 0) row_mid[i] = (uint32_t)mid;
    }
}

// Row statistics of a built network: out[0] += sum of len[0..n) (synapses),
// out[1] = max of padded[0..n) (longest padded row).
__global__ void k_row_stats(const uint64_t* len, const uint64_t* padded, const uint32_t* n1, uint32_t n,
                            unsigned long long* out) {
    unsigned long long sum = 0, mx = 0, mx1 = 0, mx2 = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        sum += len[i];
        mx = max(mx, (unsigned long long)padded[i]);
        const unsigned long long p1 = (n1[i] + kRowAlign - 1) / kRowAlign * kRowAlign;
        mx1 = max(mx1, p1);
        mx2 = max(mx2, (unsigned long long)padded[i] - p1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        mx1 = max(mx1, __shfl_xor_sync(0xFFFFFFFFu, mx1, o));
        mx2 = max(mx2, __shfl_xor_sync(0xFFFFFFFFu, mx2, o));
    }
    if ((threadIdx.x & 31u) == 0) {
        if (sum) atomicAdd(out, sum);
        if (mx) atomicMax(out + 1, mx);
        if (mx1) atomicMax(out + 3, mx1);
        if (mx2) atomicMax(out + 4, mx2);
    }
}

// Bounds of the exact-sum aggregation's fixed-point grid: in[t] += 1 for
// every synapse into storage index t, out[0] = max |w| (as bits: the order
// of non-negative floats), over the padded synapse array (padding skipped).
__global__ void k_exact_inputs(const uint32_t* tgt, const float* w, uint64_t n, uint32_t* in,
                               unsigned int* maxw_bits) {
    unsigned int mx = 0;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = tgt[j];
        if (t == kTgtSentinel) continue;
        atomicAdd(in + t, 1u);
        mx = max(mx, __float_as_uint(fabsf(w[j])));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31u) == 0 && mx) atomicMax(maxw_bits, mx);
}

// out = max of a[0..n)
__global__ void k_max_u32(const uint32_t* a, uint32_t n, unsigned int* out) {
    unsigned int mx = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) mx = max(mx, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31u) == 0 && mx) atomicMax(out, mx);
}

}  // namespace naer
