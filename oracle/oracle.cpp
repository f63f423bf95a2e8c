// ORACLE — test infrastructure only.  A CPU restatement of the reference's
// simulation step (MatteoSchmider/Naer, OpenCL C kernels under
// include/naer/kernels/ and host code src/Network.cpp), used by the tests,
// the smoke check and the CPU baseline of the benchmark as the checker.  It
// is never linked into, loaded by or called from the product library.
//
// Parity status: the reference's whole path cannot run in this environment
// (no OpenCL runtime; several included .cl files and the Random123
// submodule are not in the reference tree).  Its complete kernels
// random.cl, input_neuron_group.cl, lif.cl and network.cl are compiled as C
// under a host work-group shim (oracle/ref/, built into oracle/_ref/), and
// this restatement's Philox draws, Poisson windows, event-mode neuron
// update and Bernoulli connectivity are checked against them bit for bit
// (tests/test_ref_kernels.py, fixture tests/golden/ref_kernels.npz);
// Philox4x32-10 is also checked against cuRAND's Philox4_32_10.  The
// grid-mode semantics (fixed dt, per-synapse delays, ring aggregation, the
// configurations' pair STDP) have no counterpart in those kernels and are
// restated from the configurations ("parity unpinned" for those parts).
//
// Everything is written independently of the product sources: its own
// Philox, its own layout (reference addresses, no padding), scalar loops.
//
// Build: oracle/Makefile -> oracle/liboracle.so (g++ -O2 -fopenmp
// -ffp-contract=off; no fast-math, so fp32/fp64 operations round exactly as
// written).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11): the generator behind Random123's
// philox4x32 used at include/naer/kernels/random.cl:8-16.
void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
    }
    std::memcpy(out, c, sizeof(c));
}

}  // extern "C"

namespace {

inline void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                   uint32_t out[4]) {
    const uint32_t c[4] = {c0, c1, c2, c3};
    const uint32_t k[2] = {k0, k1};
    oracle_philox4x32_10(c, k, out);
}

// random.cl:6-24 — key {get_global_id(0), seed}, counter {iteration, 0, 0, 0},
// the third output word over UINT_MAX, as double.
inline double uniform_rand(uint32_t gid, uint32_t seed, uint32_t iteration, uint32_t* word0 = nullptr) {
    uint32_t o[4];
    philox(iteration, 0, 0, 0, gid, seed, o);
    if (word0) *word0 = o[0];
    return (double)o[2] / (double)4294967295u;
}

// random.cl:26-30 plus the (uint) cast of input_neuron_group.cl:29,37.
// x == 1.0 gives +inf; the reference's cast is undefined there, the oracle
// saturates to 0xFFFFFFFF.
inline uint32_t exp_interval_us(uint32_t gid, uint32_t seed, uint32_t iteration, double rate) {
    const double x = uniform_rand(gid, seed, iteration);
    const double dt = std::log(1.0 - x) / (-(rate / 1000000.0));
    if (!(dt < 4294967296.0)) return 0xFFFFFFFFu;
    return (uint32_t)dt;
}

// Reference work-item id of element idx of a type with groups of
// `capacity` processed by `wg` work-items (input_neuron_group.cl:17,26 with
// Network.h:110-119: Poisson capacity 2048, workgroup 128).
inline uint32_t poisson_gid(uint32_t idx) { return (idx / 2048u) * 128u + (idx % 2048u) % 128u; }

// simulate_poisson_neurons (input_neuron_group.cl:17-39) for one element.
uint32_t poisson_window(uint32_t idx, uint32_t n, uint32_t seed, double rate, uint32_t t0, uint32_t t1,
                        uint32_t* times) {
    const uint32_t gid = poisson_gid(idx);
    uint32_t time = t0 + exp_interval_us(gid, seed, t0 * n + idx, rate);
    uint32_t count = 0;
    for (uint32_t multiple = 0; multiple < 10; ++multiple) {
        if (time < t1) {
            if (times) times[count] = time;
            ++count;
            time += exp_interval_us(gid, seed, time * n + idx, rate);
        }
    }
    return count;
}

}  // namespace

extern "C" {

// exp_interval_us of generator outputs z = z_first + i * z_step (mod 2^32),
// with the host's (glibc) logarithm.
void oracle_intervals(double rate, uint32_t z_first, uint32_t z_step, uint64_t count, uint32_t* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        const uint32_t z = z_first + (uint32_t)i * z_step;
        if (z == 0xFFFFFFFFu) {
            out[i] = 0xFFFFFFFFu;
            continue;
        }
        const double x = (double)z / 4294967295.0;
        const double dt = std::log(1.0 - x) / (-(rate / 1000000.0));
        out[i] = dt < 4294967296.0 ? (uint32_t)dt : 0xFFFFFFFFu;
    }
}

double oracle_uniform_rand(uint32_t gid, uint32_t seed, uint32_t iteration) {
    return uniform_rand(gid, seed, iteration);
}

uint32_t oracle_exp_interval_us(uint32_t gid, uint32_t seed, uint32_t iteration, double rate) {
    return exp_interval_us(gid, seed, iteration, rate);
}

uint32_t oracle_poisson_window(uint32_t idx, uint32_t n, uint32_t seed, double rate, uint32_t t0,
                               uint32_t t1, uint32_t* times) {
    return poisson_window(idx, n, seed, rate, t0, t1, times);
}

// ---------------------------------------------------------------------------
// Network description (mirrors the product's C ABI parameter blocks).

struct OrPop {
    uint32_t type;  // 0 STDP, 1 NOP, 2 POISSON
    uint32_t size;
    float tau_m_ms, v_th, v_reset, t_ref_ms, v_init;
    float rate_hz, drive_rate_hz, drive_weight;
    uint32_t drive_seed, pad;
};

struct OrConn {
    uint32_t src, dst, rule, degree;  // rule 3: explicit synapses (the arrays below)
    double p;
    float weight, wmin, wmax;
    uint32_t dmin, dmax, pad;
    uint64_t seed;
    const uint64_t* rp;  // explicit: CSR over the source population (valid until the build)
    const uint32_t* tg;  // target index within the destination population
    const float* wv;
    const uint8_t* dv;
};

struct OrParams {
    uint32_t dt_us;
    uint32_t deterministic;  // 1: per-(step, cell) left fold; 0: parallel atomic adds;
                             // 2: exact sums of fixed-point weights (see exact_shift)
    uint32_t poisson_seed;
    uint32_t stdp_enabled;
    float tau_plus_ms, tau_minus_ms, a_plus, a_minus, w_max;
    uint32_t stdp_history;
    int32_t threads;  // <= 0: all available
};

}  // extern "C"

namespace {

// Event-mode state (oracle_net_run_events).
struct EvState {
    std::vector<float> v;
    std::vector<uint32_t> time;
    std::vector<std::pair<uint32_t, uint32_t>> next;  // events of the next window
    std::vector<uint32_t> sp_time, sp_id;             // raster: (µs, address)
    uint64_t window = 0, delivered = 0;
};

struct Net {
    OrParams prm{};
    std::vector<OrPop> pops;
    std::vector<OrConn> conns;
    // layout (reference addresses: Network.cpp:267-285)
    std::vector<uint32_t> base;       // address of each population's first neuron
    std::vector<uint32_t> type_addr;  // address within its type
    uint32_t n = 0, n_poisson = 0, D = 2;
    std::vector<uint8_t> kind;        // neuron type per address
    std::vector<uint32_t> pop_of;     // population per address
    // CSR in address order
    std::vector<uint64_t> row_ptr;
    std::vector<uint32_t> tgt;
    std::vector<float> w;
    std::vector<uint8_t> dly;
    // state
    std::vector<float> v;
    std::vector<uint32_t> refr;
    std::vector<float> ring;          // [D][n]
    std::vector<int32_t> ring_q;      // [D][n] exact mode: fixed-point sums, grid 2^-fx_shift
    int32_t fx_shift = 0;
    std::vector<int32_t> last_post, last_pre, hist;
    std::vector<int32_t> evicted;  // newest post spike that has left the history (-1 = none)
    std::vector<float> y_post, x_pre, e_plus, e_minus;
    uint32_t e_len = 0;
    bool plastic_on = false;
    uint64_t step = 0;
    uint64_t events = 0;
    uint64_t hist_overflow = 0;
    std::vector<uint32_t> sp_step, sp_id;
    std::vector<float> partial;
    std::vector<uint8_t> touched_flag;
    std::vector<uint64_t> touched;
    std::unique_ptr<EvState> ev;  // event-mode state (oracle_net_run_events)
};

inline uint32_t pick(uint32_t word, uint32_t n) { return (uint32_t)(((uint64_t)word * n) >> 32); }

inline uint32_t delay_of(const OrConn& c, uint32_t word) {
    if (c.dmax <= c.dmin) return c.dmin;
    return c.dmin + pick(word, c.dmax - c.dmin + 1);
}

inline float uniform_weight(float wmin, float wmax, float x) {
    const float span = wmax - wmin;
    const float prod = span * x;
    return wmin + prod;
}

inline float unit_float(uint32_t word) { return (float)(word >> 8) * (1.0f / 16777216.0f); }

void layout(Net& net) {
    uint32_t count[3] = {0, 0, 0};
    net.type_addr.resize(net.pops.size());
    for (size_t i = 0; i < net.pops.size(); ++i) {
        net.type_addr[i] = count[net.pops[i].type];
        count[net.pops[i].type] += net.pops[i].size;
    }
    const uint32_t type_base[3] = {0, count[0], count[0] + count[1]};
    net.n = count[0] + count[1] + count[2];
    net.n_poisson = count[2];
    net.base.resize(net.pops.size());
    net.kind.assign(net.n, 0);
    net.pop_of.assign(net.n, 0);
    for (size_t i = 0; i < net.pops.size(); ++i) {
        net.base[i] = type_base[net.pops[i].type] + net.type_addr[i];
        for (uint32_t k = 0; k < net.pops[i].size; ++k) {
            net.kind[net.base[i] + k] = (uint8_t)net.pops[i].type;
            net.pop_of[net.base[i] + k] = (uint32_t)i;
        }
    }
    uint32_t dmax = 1;
    for (const auto& c : net.conns) dmax = std::max(dmax, c.dmax);
    net.D = dmax + 1;
}

// Connectivity.  Rows: connections in declaration order; within a
// connection REF_BERNOULLI by ascending target, FIXED_OUTDEGREE by draw k,
// FIXED_INDEGREE by ascending (target, k); then a stable partition puts the
// delay-1 synapses first.  Two passes: per-(connection, source) counts, then
// the fill at prefix-sum offsets.
void build_csr(Net& net) {
    const size_t nc = net.conns.size();
    std::vector<std::vector<uint32_t>> cnt(nc);
    // pass 1: counts
    for (size_t ci = 0; ci < nc; ++ci) {
        const OrConn& c = net.conns[ci];
        const OrPop& sp = net.pops[c.src];
        const OrPop& dp = net.pops[c.dst];
        const uint32_t seed_lo = (uint32_t)c.seed, seed_hi = (uint32_t)(c.seed >> 32);
        cnt[ci].assign(sp.size, 0);
        if (c.rule == 0) {
            // count_connections (network.cl:14-49): the test for (s, d) runs on
            // work-item s*32 + d%32 with counter d.
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t s = 0; s < (int64_t)sp.size; ++s) {
                uint32_t k = 0;
                for (uint32_t d = 0; d < dp.size; ++d)
                    if (uniform_rand((uint32_t)s * 32u + d % 32u, seed_lo, d) < c.p) ++k;
                cnt[ci][s] = k;
            }
        } else if (c.rule == 2) {
            std::fill(cnt[ci].begin(), cnt[ci].end(), c.degree);
        } else if (c.rule == 3) {
            for (uint32_t s = 0; s < sp.size; ++s) cnt[ci][s] = (uint32_t)(c.rp[s + 1] - c.rp[s]);
        } else {
            for (uint32_t i = 0; i < dp.size; ++i)
                for (uint32_t b = 0; b < (c.degree + 3) / 4; ++b) {
                    uint32_t os[4];
                    philox(i, b, 0, 0, seed_lo, seed_hi, os);
                    for (uint32_t j = 0; j < 4 && b * 4 + j < c.degree; ++j) ++cnt[ci][pick(os[j], sp.size)];
                }
        }
    }
    net.row_ptr.assign(net.n + 1, 0);
    for (size_t ci = 0; ci < nc; ++ci) {
        const uint32_t sb = net.base[net.conns[ci].src];
        for (uint32_t s = 0; s < cnt[ci].size(); ++s) net.row_ptr[sb + s + 1] += cnt[ci][s];
    }
    for (uint32_t i = 0; i < net.n; ++i) net.row_ptr[i + 1] += net.row_ptr[i];
    const uint64_t S = net.row_ptr[net.n];
    net.tgt.resize(S);
    net.w.resize(S);
    net.dly.resize(S);
    std::vector<uint64_t> cur(net.row_ptr.begin(), net.row_ptr.end() - 1);
    // pass 2: fill
    for (size_t ci = 0; ci < nc; ++ci) {
        const OrConn& c = net.conns[ci];
        const OrPop& sp = net.pops[c.src];
        const OrPop& dp = net.pops[c.dst];
        const uint32_t sb = net.base[c.src], db = net.base[c.dst];
        const uint32_t seed_lo = (uint32_t)c.seed, seed_hi = (uint32_t)(c.seed >> 32);
        if (c.rule == 0) {
            // generate_connections (network.cl:63-107); weight 0 => random
            // weight from the same draw (network.cl:97-100)
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t s = 0; s < (int64_t)sp.size; ++s) {
                uint64_t o = cur[sb + s];
                for (uint32_t d = 0; d < dp.size; ++d) {
                    uint32_t word0 = 0;
                    const double x = uniform_rand((uint32_t)s * 32u + d % 32u, seed_lo, d, &word0);
                    if (!(x < c.p)) continue;
                    net.tgt[o] = db + d;
                    net.w[o] = c.weight == 0.0f ? uniform_weight(c.wmin, c.wmax, (float)x) : c.weight;
                    net.dly[o] = (uint8_t)delay_of(c, word0);
                    ++o;
                }
            }
        } else if (c.rule == 3) {
            // explicit synapses, each row in the given order
            for (uint32_t s = 0; s < sp.size; ++s)
                for (uint64_t j = c.rp[s]; j < c.rp[s + 1]; ++j) {
                    const uint64_t q = cur[sb + s] + (j - c.rp[s]);
                    net.tgt[q] = db + c.tg[j];
                    net.w[q] = c.wv[j];
                    net.dly[q] = c.dv[j];
                }
        } else if (c.rule == 2) {
#pragma omp parallel for schedule(static)
            for (int64_t s = 0; s < (int64_t)sp.size; ++s) {
                const uint64_t o = cur[sb + s];
                for (uint32_t b = 0; b < (c.degree + 3) / 4; ++b) {
                    uint32_t ot[4], od[4], ow[4] = {0, 0, 0, 0};
                    philox((uint32_t)s, b, 0, 0, seed_lo, seed_hi, ot);
                    philox((uint32_t)s, b, 1, 0, seed_lo, seed_hi, od);
                    if (c.weight == 0.0f) philox((uint32_t)s, b, 2, 0, seed_lo, seed_hi, ow);
                    for (uint32_t j = 0; j < 4 && b * 4 + j < c.degree; ++j) {
                        const uint64_t q = o + b * 4 + j;
                        net.tgt[q] = db + pick(ot[j], dp.size);
                        net.w[q] = c.weight == 0.0f ? uniform_weight(c.wmin, c.wmax, unit_float(ow[j])) : c.weight;
                        net.dly[q] = (uint8_t)delay_of(c, od[j]);
                    }
                }
            }
        } else {
            std::vector<uint64_t> pos(sp.size);
            for (uint32_t s = 0; s < sp.size; ++s) pos[s] = cur[sb + s];
            for (uint32_t i = 0; i < dp.size; ++i)
                for (uint32_t b = 0; b < (c.degree + 3) / 4; ++b) {
                    uint32_t os[4], od[4], ow[4] = {0, 0, 0, 0};
                    philox(i, b, 0, 0, seed_lo, seed_hi, os);
                    philox(i, b, 1, 0, seed_lo, seed_hi, od);
                    if (c.weight == 0.0f) philox(i, b, 2, 0, seed_lo, seed_hi, ow);
                    for (uint32_t j = 0; j < 4 && b * 4 + j < c.degree; ++j) {
                        const uint64_t q = pos[pick(os[j], sp.size)]++;
                        net.tgt[q] = db + i;
                        net.w[q] = c.weight == 0.0f ? uniform_weight(c.wmin, c.wmax, unit_float(ow[j])) : c.weight;
                        net.dly[q] = (uint8_t)delay_of(c, od[j]);
                    }
                }
        }
        for (uint32_t s = 0; s < sp.size; ++s) cur[sb + s] += cnt[ci][s];
    }
    // Canonical row order: a stable partition that puts the synapses of
    // delay 1 (the ones the next step needs) before the others.
    std::vector<uint32_t> tt;
    std::vector<float> ww;
    std::vector<uint8_t> dd;
    for (uint32_t i = 0; i < net.n; ++i) {
        const uint64_t b = net.row_ptr[i], e = net.row_ptr[i + 1];
        tt.clear();
        ww.clear();
        dd.clear();
        for (int pass = 0; pass < 2; ++pass)
            for (uint64_t j = b; j < e; ++j)
                if ((net.dly[j] == 1) == (pass == 0)) {
                    tt.push_back(net.tgt[j]);
                    ww.push_back(net.w[j]);
                    dd.push_back(net.dly[j]);
                }
        std::copy(tt.begin(), tt.end(), net.tgt.begin() + b);
        std::copy(ww.begin(), ww.end(), net.w.begin() + b);
        std::copy(dd.begin(), dd.end(), net.dly.begin() + b);
    }
}

// Exact-sum aggregation: every delivered weight (after STDP and the POISSON
// multiplicity) becomes the integer nearest to w * 2^S and the ring holds
// int32 sums, which no summation order changes; the neuron reads a cell as
// float(sum) * 2^-S.  S is the largest shift (at most 30) for which no cell
// sum can overflow: a cell receives at most one event per synapse into its
// neuron before it is read, each of magnitude at most max|w| (w_max for a
// plastic net) times 10 (the largest POISSON multiplicity), plus half a unit
// of rounding.  Returns -1 when even S = 0 cannot hold that bound.
int32_t exact_shift(const Net& net) {
    std::vector<uint32_t> in(net.n, 0);
    float maxw = 0.0f;
    for (size_t j = 0; j < net.tgt.size(); ++j) {
        ++in[net.tgt[j]];
        maxw = std::max(maxw, std::fabs(net.w[j]));
    }
    uint32_t max_in = 0;
    for (uint32_t c : in) max_in = std::max(max_in, c);
    if (net.plastic_on) maxw = std::max(maxw, net.prm.w_max);
    bool poisson = false;
    for (const OrPop& p : net.pops) poisson = poisson || (p.type == 2 && p.size > 0);
    const double bound = (double)max_in * (double)maxw * (poisson ? 10.0 : 1.0);
    for (int32_t S = 30; S >= 0; --S)
        if (bound * std::ldexp(1.0, S) + (double)max_in <= 2147483647.0) return S;
    return -1;
}

void init_state(Net& net) {
    net.v.assign(net.n, 0.0f);
    net.refr.assign(net.n, 0);
    for (size_t p = 0; p < net.pops.size(); ++p)
        if (net.pops[p].type != 2)
            for (uint32_t k = 0; k < net.pops[p].size; ++k) net.v[net.base[p] + k] = net.pops[p].v_init;
    net.ring.assign((size_t)net.D * net.n, 0.0f);
    if (net.prm.deterministic == 2) net.ring_q.assign((size_t)net.D * net.n, 0);
    const OrParams& P = net.prm;
    uint32_t n_stdp = 0;
    for (const auto& p : net.pops)
        if (p.type == 0) n_stdp += p.size;
    net.plastic_on = P.stdp_enabled && n_stdp > 0;
    if (net.plastic_on) {
        net.last_post.assign(net.n, -1);
        net.evicted.assign(net.n, -1);
        net.last_pre.assign(net.n, -1);
        net.y_post.assign(net.n, 0.0f);
        net.x_pre.assign(net.n, 0.0f);
        net.hist.assign((size_t)net.n * P.stdp_history, -1);
        const double tmax = std::max((double)P.tau_plus_ms, (double)P.tau_minus_ms) * 1000.0;
        net.e_len = (uint32_t)std::min<double>(std::ceil(104.0 * tmax / P.dt_us) + 1.0, 1 << 24);
        net.e_plus.resize(net.e_len);
        net.e_minus.resize(net.e_len);
        for (uint32_t k = 0; k < net.e_len; ++k) {
            net.e_plus[k] = (float)std::exp(-(double)k * P.dt_us / ((double)P.tau_plus_ms * 1000.0));
            net.e_minus[k] = (float)std::exp(-(double)k * P.dt_us / ((double)P.tau_minus_ms * 1000.0));
        }
    }
    net.partial.assign((size_t)net.D * net.n, 0.0f);
    net.touched_flag.assign((size_t)net.D * net.n, 0);
}

inline float decay(const std::vector<float>& tab, int64_t k) {
    return (k >= 0 && (uint64_t)k < tab.size()) ? tab[(size_t)k] : 0.0f;
}

struct Spike {
    uint32_t src;
    int32_t pre_last;  // STDP sources: previous pre spike step; POISSON: multiplicity
    float pre_x;
};

// Pair-based STDP at the pre spike of step t: lazy LTP over the post spikes
// of tgt in (pre_last, t], oldest first, then LTD with the post trace at t;
// clip to [0, w_max] after every update.
float stdp(Net& net, float wv, uint32_t tgt, int32_t t, int32_t pre_last, float pre_x, uint64_t& ovf) {
    const OrParams& P = net.prm;
    const float ap = P.a_plus * P.w_max;
    const float am = P.a_minus * P.w_max;
    if (pre_last >= 0) {
        const int32_t* h = &net.hist[(size_t)tgt * P.stdp_history];
        uint32_t c = 0;
        while (c < P.stdp_history && h[c] > pre_last) ++c;
        // lost pairs: a post spike that left the history still falls after pre_last
        if (c == P.stdp_history && net.evicted[tgt] > pre_last) ++ovf;
        for (int k = (int)c - 1; k >= 0; --k) {
            const float x = pre_x * decay(net.e_plus, h[k] - pre_last);
            const float inc = ap * x;
            wv = std::min(wv + inc, P.w_max);
        }
    }
    const int32_t lp = net.last_post[tgt];
    if (lp >= 0) {
        const float y = net.y_post[tgt] * decay(net.e_minus, t - lp);
        const float dec = am * y;
        wv = std::max(wv - dec, 0.0f);
    }
    return wv;
}

// One grid step (dt = prm.dt_us): neuron update for every address, then the
// scatter of this step's spikes into the ring.  Returns nothing; spikes are
// appended to sp_step/sp_id.
void grid_step(Net& net) {
    const OrParams& P = net.prm;
    const uint32_t t = (uint32_t)net.step;
    const uint32_t slot = t % net.D;
    const uint32_t t0 = t * P.dt_us, t1 = t0 + P.dt_us;
    const int nthreads =
#ifdef _OPENMP
        P.threads > 0 ? P.threads : omp_get_max_threads();
#else
        1;
#endif
    std::vector<std::vector<Spike>> per_thread(nthreads);
    std::vector<double> prop(net.pops.size());
    std::vector<uint32_t> tref(net.pops.size());
    for (size_t p = 0; p < net.pops.size(); ++p) {
        prop[p] = std::exp(-(double)P.dt_us / ((double)net.pops[p].tau_m_ms * 1000.0));
        tref[p] = (uint32_t)std::llround((double)net.pops[p].t_ref_ms * 1000.0 / P.dt_us);
    }
    float* ring_slot = &net.ring[(size_t)slot * net.n];

#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        std::vector<Spike>& out = per_thread[tid];
#pragma omp for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)net.n; ++ii) {
            const uint32_t i = (uint32_t)ii;
            const uint32_t pi = net.pop_of[i];
            const OrPop& pop = net.pops[pi];
            if (pop.type == 2) {
                if (!(pop.rate_hz > 0.0f)) continue;
                const uint32_t idx = net.type_addr[pi] + (i - net.base[pi]);
                const uint32_t m = poisson_window(idx, net.n_poisson, P.poisson_seed, (double)pop.rate_hz, t0, t1,
                                                  nullptr);
                if (m) out.push_back(Spike{i, (int32_t)m, 0.0f});
                continue;
            }
            float I;
            if (P.deterministic == 2) {
                int32_t& q = net.ring_q[(size_t)slot * net.n + i];
                I = (float)q * std::ldexp(1.0f, -net.fx_shift);
                q = 0;
            } else {
                I = ring_slot[i];
                ring_slot[i] = 0.0f;
            }
            if (net.refr[i] > 0) {
                net.refr[i] -= 1;
                continue;
            }
            // decay, ring input and drive in double, one rounding to fp32
            double x = (double)net.v[i] * prop[pi];
            x = x + (double)I;
            if (pop.drive_rate_hz > 0.0f) {
                const uint32_t m = poisson_window(i - net.base[pi], pop.size, pop.drive_seed,
                                                  (double)pop.drive_rate_hz, t0, t1, nullptr);
                if (m) x = x + (double)m * (double)pop.drive_weight;
            }
            float v = (float)x;
            if (v > pop.v_th) {
                v = pop.v_reset;
                net.refr[i] = tref[pi];
                Spike sp{i, 0, 0.0f};
                if (net.plastic_on && pop.type == 0) {
                    const int32_t ts = (int32_t)t;
                    const int32_t lp = net.last_post[i];
                    const float y = lp >= 0 ? net.y_post[i] * decay(net.e_minus, ts - lp) : 0.0f;
                    net.y_post[i] = y + 1.0f;
                    net.last_post[i] = ts;
                    int32_t* h = &net.hist[(size_t)i * P.stdp_history];
                    if (h[P.stdp_history - 1] >= 0) net.evicted[i] = h[P.stdp_history - 1];
                    for (int k = (int)P.stdp_history - 1; k > 0; --k) h[k] = h[k - 1];
                    h[0] = ts;
                    sp.pre_last = net.last_pre[i];
                    sp.pre_x = net.x_pre[i];
                    const float x = sp.pre_last >= 0 ? net.x_pre[i] * decay(net.e_plus, ts - sp.pre_last) : 0.0f;
                    net.x_pre[i] = x + 1.0f;
                    net.last_pre[i] = ts;
                }
                out.push_back(sp);
            }
            net.v[i] = v;
        }
    }
    // spikes in ascending address order (static schedule keeps chunks ordered)
    std::vector<Spike> spikes;
    for (auto& pt : per_thread) spikes.insert(spikes.end(), pt.begin(), pt.end());
    for (const auto& sp : spikes) {
        net.sp_step.push_back(t);
        net.sp_id.push_back(sp.src);
    }

    const uint32_t tmod = t % net.D;
    uint64_t ev = 0, ovf = 0;
    auto deliver_weight = [&](const Spike& sp, uint64_t j) -> float {
        float wv = net.w[j];
        const uint32_t tg = net.tgt[j];
        const bool src_plastic = net.plastic_on && net.kind[sp.src] == 0;
        if (src_plastic && net.kind[tg] == 0) {
            wv = stdp(net, wv, tg, (int32_t)t, sp.pre_last, sp.pre_x, ovf);
            net.w[j] = wv;
        }
        if (!src_plastic && sp.pre_last > 1) wv = wv * (float)sp.pre_last;
        return wv;
    };
    auto cell_of = [&](uint64_t j) -> uint64_t {
        uint32_t sl = tmod + net.dly[j];
        if (sl >= net.D) sl -= net.D;
        return (uint64_t)sl * net.n + net.tgt[j];
    };

    if (P.deterministic == 2) {
        // exact sums: integer additions in any order
        const float scale = std::ldexp(1.0f, net.fx_shift);
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : ev, ovf) num_threads(nthreads)
        for (int64_t si = 0; si < (int64_t)spikes.size(); ++si) {
            const Spike& sp = spikes[(size_t)si];
            uint64_t local_ovf = 0;
            for (uint64_t j = net.row_ptr[sp.src]; j < net.row_ptr[sp.src + 1]; ++j) {
                float wv = net.w[j];
                const uint32_t tg = net.tgt[j];
                const bool src_plastic = net.plastic_on && net.kind[sp.src] == 0;
                if (src_plastic && net.kind[tg] == 0) {
                    wv = stdp(net, wv, tg, (int32_t)t, sp.pre_last, sp.pre_x, local_ovf);
                    net.w[j] = wv;
                }
                if (!src_plastic && sp.pre_last > 1) wv = wv * (float)sp.pre_last;
                const int32_t q = (int32_t)std::nearbyint(wv * scale);
                std::atomic_ref<int32_t>(net.ring_q[cell_of(j)]).fetch_add(q, std::memory_order_relaxed);
                ++ev;
            }
            ovf += local_ovf;
        }
    } else if (P.deterministic) {
        // per (step, cell): left fold in (source, synapse) order, then add
        for (const auto& sp : spikes) {
            for (uint64_t j = net.row_ptr[sp.src]; j < net.row_ptr[sp.src + 1]; ++j) {
                const float wv = deliver_weight(sp, j);
                const uint64_t cell = cell_of(j);
                if (!net.touched_flag[cell]) {
                    net.touched_flag[cell] = 1;
                    net.touched.push_back(cell);
                    net.partial[cell] = wv;
                } else {
                    net.partial[cell] = net.partial[cell] + wv;
                }
                ++ev;
            }
        }
        for (uint64_t cell : net.touched) {
            net.ring[cell] = net.ring[cell] + net.partial[cell];
            net.touched_flag[cell] = 0;
        }
        net.touched.clear();
    } else {
        // the multithreaded baseline: spikes in parallel, atomic float adds
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : ev, ovf) num_threads(nthreads)
        for (int64_t si = 0; si < (int64_t)spikes.size(); ++si) {
            const Spike& sp = spikes[(size_t)si];
            uint64_t local_ovf = 0;
            for (uint64_t j = net.row_ptr[sp.src]; j < net.row_ptr[sp.src + 1]; ++j) {
                float wv = net.w[j];
                const uint32_t tg = net.tgt[j];
                const bool src_plastic = net.plastic_on && net.kind[sp.src] == 0;
                if (src_plastic && net.kind[tg] == 0) {
                    wv = stdp(net, wv, tg, (int32_t)t, sp.pre_last, sp.pre_x, local_ovf);
                    net.w[j] = wv;
                }
                if (!src_plastic && sp.pre_last > 1) wv = wv * (float)sp.pre_last;
                std::atomic_ref<float>(net.ring[cell_of(j)]).fetch_add(wv, std::memory_order_relaxed);
                ++ev;
            }
            ovf += local_ovf;
        }
    }
    net.events += ev;
    net.hist_overflow += ovf;
    ++net.step;
}

}  // namespace

extern "C" {

void* oracle_net_create(const OrParams* prm, const OrPop* pops, uint32_t npops, const OrConn* conns,
                        uint32_t nconns) {
    Net* net = new Net();
    net->prm = *prm;
    net->pops.assign(pops, pops + npops);
    net->conns.assign(conns, conns + nconns);
    layout(*net);
    return net;
}

void oracle_net_destroy(void* h) { delete static_cast<Net*>(h); }

int oracle_net_build(void* h) {
    Net& net = *static_cast<Net*>(h);
    build_csr(net);
    init_state(net);
    if (net.prm.deterministic == 2) {
        net.fx_shift = exact_shift(net);
        if (net.fx_shift < 0) return -1;
    }
    return 0;
}

int32_t oracle_net_exact_shift(void* h) { return static_cast<Net*>(h)->fx_shift; }

uint32_t oracle_net_neurons(void* h) { return static_cast<Net*>(h)->n; }
uint64_t oracle_net_synapses(void* h) { return static_cast<Net*>(h)->tgt.size(); }
uint32_t oracle_net_ring_slots(void* h) { return static_cast<Net*>(h)->D; }
uint32_t oracle_net_population_base(void* h, uint32_t pop) { return static_cast<Net*>(h)->base[pop]; }

void oracle_net_copy_csr(void* h, uint64_t* row_ptr, uint32_t* tgt, float* w, uint8_t* d) {
    const Net& net = *static_cast<Net*>(h);
    std::copy(net.row_ptr.begin(), net.row_ptr.end(), row_ptr);
    if (tgt) std::copy(net.tgt.begin(), net.tgt.end(), tgt);
    if (w) std::copy(net.w.begin(), net.w.end(), w);
    if (d) std::copy(net.dly.begin(), net.dly.end(), d);
}

// Replace weights (address-order CSR) before running, e.g. with the
// product's own arrays.
void oracle_net_set_weights(void* h, const float* w) {
    Net& net = *static_cast<Net*>(h);
    std::copy(w, w + net.w.size(), net.w.begin());
}

int oracle_net_run(void* h, uint64_t nsteps) {
    Net& net = *static_cast<Net*>(h);
    for (uint64_t k = 0; k < nsteps; ++k) grid_step(net);
    return 0;
}

uint64_t oracle_net_step(void* h) { return static_cast<Net*>(h)->step; }
uint64_t oracle_net_events(void* h) { return static_cast<Net*>(h)->events; }
uint64_t oracle_net_hist_overflow(void* h) { return static_cast<Net*>(h)->hist_overflow; }
uint64_t oracle_net_spike_count(void* h) { return static_cast<Net*>(h)->sp_id.size(); }

void oracle_net_copy_spikes(void* h, uint32_t* steps, uint32_t* ids) {
    const Net& net = *static_cast<Net*>(h);
    std::copy(net.sp_step.begin(), net.sp_step.end(), steps);
    std::copy(net.sp_id.begin(), net.sp_id.end(), ids);
}

void oracle_net_clear_spikes(void* h) {
    Net& net = *static_cast<Net*>(h);
    net.sp_step.clear();
    net.sp_id.clear();
}

void oracle_net_copy_state(void* h, float* v, uint32_t* refr) {
    const Net& net = *static_cast<Net*>(h);
    for (uint32_t i = 0; i < net.n; ++i) {
        const bool lif = net.kind[i] != 2;
        if (v) v[i] = lif ? net.v[i] : 0.0f;
        if (refr) refr[i] = lif ? net.refr[i] : 0u;
    }
}

void oracle_net_set_state(void* h, const float* v, const uint32_t* refr) {
    Net& net = *static_cast<Net*>(h);
    for (uint32_t i = 0; i < net.n; ++i) {
        if (net.kind[i] == 2) continue;
        if (v) net.v[i] = v[i];
        if (refr) net.refr[i] = refr[i];
    }
}

void oracle_net_copy_ring(void* h, float* ring) {
    const Net& net = *static_cast<Net*>(h);
    if (net.prm.deterministic == 2) std::memcpy(ring, net.ring_q.data(), net.ring_q.size() * 4);  // the sums' bits
    else std::copy(net.ring.begin(), net.ring.end(), ring);
}

void oracle_net_copy_weights(void* h, float* w) {
    const Net& net = *static_cast<Net*>(h);
    std::copy(net.w.begin(), net.w.end(), w);
}

int oracle_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// FP64 re-integration of a finished run.  The network restarts from its
// initial state and every arithmetic step is done in double, with exact
// exp() decay factors, but the spike times are the run's own (its raster),
// not recomputed from thresholds: this is the trajectory the run's fp32
// arithmetic approximates for the same spike inputs.  A POISSON source's
// multiplicity and every drive count come from the same Poisson windows.
// Outputs the final membrane potentials (address order) and the final
// weights (address-order CSR, as oracle_net_copy_weights); *mismatch counts
// (step, neuron) pairs where the double trajectory's threshold test
// disagrees with the raster (V > V_th without a recorded spike, or a
// recorded spike while refractory), a diagnostic only.
// uncapped != 0: lazy LTP sees every post spike since the source's last
// spike (the pair rule without the post-history limit the device and the
// fp32 oracle share); *lost counts, with the limit, the pairs it drops.
int oracle_reintegrate_fp64_ex(void* h, uint64_t nsteps, const uint32_t* sp_step, const uint32_t* sp_id, uint64_t nsp,
                               double* v_out, double* w_out, uint64_t* mismatch, int uncapped, uint64_t* lost) {
    const Net& net = *static_cast<Net*>(h);
    const OrParams& P = net.prm;
    std::vector<std::vector<int32_t>> posts;  // every post spike, oldest first (uncapped)
    uint64_t dropped = 0;
    const uint32_t n = net.n, D = net.D;
    std::vector<double> v(n, 0.0), ring((size_t)D * n, 0.0), w(net.w.begin(), net.w.end());
    std::vector<uint32_t> refr(n, 0);
    for (size_t p = 0; p < net.pops.size(); ++p)
        if (net.pops[p].type != 2)
            for (uint32_t k = 0; k < net.pops[p].size; ++k) v[net.base[p] + k] = net.pops[p].v_init;
    uint32_t n_stdp = 0;
    for (const auto& p : net.pops)
        if (p.type == 0) n_stdp += p.size;
    const bool plastic = P.stdp_enabled && n_stdp > 0;
    std::vector<int32_t> last_post(n, -1), last_pre(n, -1), hist(plastic ? (size_t)n * P.stdp_history : 0, -1);
    std::vector<double> y_post(n, 0.0), x_pre(n, 0.0);
    const double tau_p = (double)P.tau_plus_ms * 1000.0, tau_m = (double)P.tau_minus_ms * 1000.0;
    const double ap = (double)P.a_plus * P.w_max, am = (double)P.a_minus * P.w_max, wmax = P.w_max;
    std::vector<double> prop(net.pops.size());
    std::vector<uint32_t> tref(net.pops.size());
    for (size_t p = 0; p < net.pops.size(); ++p) {
        prop[p] = std::exp(-(double)P.dt_us / ((double)net.pops[p].tau_m_ms * 1000.0));
        tref[p] = (uint32_t)std::llround((double)net.pops[p].t_ref_ms * 1000.0 / P.dt_us);
    }
    std::vector<uint8_t> fired(n, 0);
    uint64_t mis = 0, k = 0;
    for (uint64_t t = 0; t < nsteps; ++t) {
        const uint32_t t0 = (uint32_t)t * P.dt_us, t1 = t0 + P.dt_us;
        const uint32_t slot = (uint32_t)(t % D);
        std::vector<uint32_t> spk;
        while (k < nsp && sp_step[k] < t) ++k;
        while (k < nsp && sp_step[k] == t) {
            if (sp_id[k] < n) {
                fired[sp_id[k]] = 1;
                spk.push_back(sp_id[k]);
            }
            ++k;
        }
        std::vector<uint32_t> mult(spk.size(), 1);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t pi = net.pop_of[i];
            const OrPop& pop = net.pops[pi];
            if (pop.type == 2) continue;
            const double I = ring[(size_t)slot * n + i];
            ring[(size_t)slot * n + i] = 0.0;
            if (refr[i] > 0) {
                refr[i] -= 1;
                if (fired[i]) ++mis;
                continue;
            }
            double x = v[i] * prop[pi] + I;
            if (pop.drive_rate_hz > 0.0f) {
                const uint32_t m = poisson_window(i - net.base[pi], pop.size, pop.drive_seed,
                                                  (double)pop.drive_rate_hz, t0, t1, nullptr);
                x += (double)m * (double)pop.drive_weight;
            }
            if (fired[i]) {
                x = pop.v_reset;
                refr[i] = tref[pi];
                if (plastic && pop.type == 0) {
                    const int32_t ts = (int32_t)t;
                    const int32_t lp = last_post[i];
                    const double y = lp >= 0 ? y_post[i] * std::exp(-(double)(ts - lp) * P.dt_us / tau_m) : 0.0;
                    y_post[i] = y + 1.0;
                    last_post[i] = ts;
                    int32_t* hh = &hist[(size_t)i * P.stdp_history];
                    for (int q = (int)P.stdp_history - 1; q > 0; --q) hh[q] = hh[q - 1];
                    hh[0] = ts;
                    if (posts.empty()) posts.resize(n);
                    posts[i].push_back(ts);
                }
            } else if (x > (double)pop.v_th) {
                ++mis;
            }
            v[i] = x;
        }
        // pre state before this step's spikes, for the lazy STDP of their rows
        std::vector<int32_t> pre_last(spk.size(), -1);
        std::vector<double> pre_x(spk.size(), 0.0);
        for (size_t a = 0; a < spk.size(); ++a) {
            const uint32_t i = spk[a];
            const OrPop& pop = net.pops[net.pop_of[i]];
            if (pop.type == 2) {
                const uint32_t idx = net.type_addr[net.pop_of[i]] + (i - net.base[net.pop_of[i]]);
                mult[a] = poisson_window(idx, net.n_poisson, P.poisson_seed, (double)pop.rate_hz, t0, t1, nullptr);
            } else if (plastic && pop.type == 0) {
                const int32_t ts = (int32_t)t;
                pre_last[a] = last_pre[i];
                pre_x[a] = x_pre[i];
                const double x = last_pre[i] >= 0 ? x_pre[i] * std::exp(-(double)(ts - last_pre[i]) * P.dt_us / tau_p) : 0.0;
                x_pre[i] = x + 1.0;
                last_pre[i] = ts;
            }
        }
        for (size_t a = 0; a < spk.size(); ++a) {
            const uint32_t src = spk[a];
            const bool src_plastic = plastic && net.kind[src] == 0;
            for (uint64_t j = net.row_ptr[src]; j < net.row_ptr[src + 1]; ++j) {
                const uint32_t tg = net.tgt[j];
                double wv = w[j];
                if (src_plastic && net.kind[tg] == 0) {
                    if (pre_last[a] >= 0) {
                        // post spikes in (pre_last, t], oldest first
                        static const std::vector<int32_t> none;
                        const std::vector<int32_t>& all = posts.empty() ? none : posts[tg];
                        size_t first = all.size();
                        while (first > 0 && all[first - 1] > pre_last[a]) --first;
                        const size_t avail = all.size() - first;
                        const size_t keep = std::min<size_t>(avail, P.stdp_history);
                        dropped += avail - keep;
                        for (size_t q = uncapped ? first : all.size() - keep; q < all.size(); ++q) {
                            const double xx = pre_x[a] * std::exp(-(double)(all[q] - pre_last[a]) * P.dt_us / tau_p);
                            wv = std::min(wv + ap * xx, wmax);
                        }
                    }
                    if (last_post[tg] >= 0) {
                        const double y = y_post[tg] * std::exp(-(double)((int32_t)t - last_post[tg]) * P.dt_us / tau_m);
                        wv = std::max(wv - am * y, 0.0);
                    }
                    w[j] = wv;
                }
                const double dv = src_plastic ? wv : wv * (double)mult[a];
                uint32_t sl = slot + net.dly[j];
                if (sl >= D) sl -= D;
                ring[(size_t)sl * n + tg] += dv;
            }
        }
        for (uint32_t i : spk) fired[i] = 0;
    }
    if (v_out) std::copy(v.begin(), v.end(), v_out);
    if (w_out) std::copy(w.begin(), w.end(), w_out);
    if (mismatch) *mismatch = mis;
    if (lost) *lost = dropped;
    return 0;
}

int oracle_reintegrate_fp64(void* h, uint64_t nsteps, const uint32_t* sp_step, const uint32_t* sp_id, uint64_t nsp,
                            double* v_out, double* w_out, uint64_t* mismatch) {
    return oracle_reintegrate_fp64_ex(h, nsteps, sp_step, sp_id, nsp, v_out, w_out, mismatch, 0, nullptr);
}

// ---------------------------------------------------------------------------
// Reference-compatible event mode (the `.cl` kernels' own time model).
//
// Time is continuous in µs and advances in windows of 1500 µs
// (src/Network.cpp:124-127).  Every spike is an event (arrival time, source):
// a POISSON source's events are its spike times (input_neuron_group.cl:29-38,
// generated for the window they fall in), a LIF neuron's spike at input time
// T arrives at its targets at T + 1500 µs (NAER_AXONAL_DELAY, naer_types.h:4;
// nop.cl:76), i.e. in the next window.  A window's events are applied in
// time order (ties: ascending source address — the reference's order comes
// from its scatter and is not defined), each delivering its row to its
// LIF targets through neuron_dynamics (lif.cl:15-34): dt = T - time; inputs
// with dt < 0 (refractory) are dropped; V = fp32(fp64(V) * exp(-dt / tau));
// V += w; time = T; V > V_th -> spike, time += t_ref, V = V_reset.  The
// per-population tau_m, t_ref, V_th, V_reset replace lif.cl's constants
// (20 ms, 2 ms, 20 mV, 0).  Connection delays, LIF drive and plasticity do
// not exist in this model and are ignored (the reference's STDP kernel is
// partially undefined: NAER_STDP_WEIGHT is never defined, stdp.cl:100).
//
// flags bit 0 reproduces nop.cl:54-55: per (spike, 512-neuron NOP group) only
// the first 96 synapses (the NOP workgroup size, Network.h:115-119) are
// delivered; STDP targets loop over all synapses (stdp.cl:88-92).
// Runs nwin more windows of the event model on a built network.  The event
// state lives beside the grid state of the same handle; the first call
// starts it from the initial potentials.
int oracle_net_run_events(void* h, uint64_t nwin, uint32_t flags) {
    Net& net = *static_cast<Net*>(h);
    const OrParams& P = net.prm;
    if (!net.ev) {
        net.ev = std::make_unique<EvState>();
        net.ev->v.assign(net.n, 0.0f);
        net.ev->time.assign(net.n, 0u);
        for (size_t p = 0; p < net.pops.size(); ++p)
            if (net.pops[p].type != 2)
                for (uint32_t k = 0; k < net.pops[p].size; ++k) net.ev->v[net.base[p] + k] = net.pops[p].v_init;
    }
    EvState& E = *net.ev;
    uint32_t count[3] = {0, 0, 0};
    for (const auto& p : net.pops) count[p.type] += p.size;
    const uint32_t nop_base = count[0];
    const uint32_t W = 1500;
    std::vector<uint32_t> seg_count;
    for (uint64_t k = 0; k < nwin; ++k) {
        const uint32_t t0 = (uint32_t)(E.window * W), t1 = t0 + W;
        std::vector<std::pair<uint32_t, uint32_t>> ev;
        ev.swap(E.next);
        uint32_t times[10];
        for (size_t p = 0; p < net.pops.size(); ++p) {
            const OrPop& pop = net.pops[p];
            if (pop.type != 2 || !(pop.rate_hz > 0.0f)) continue;
            for (uint32_t i = 0; i < pop.size; ++i) {
                const uint32_t idx = net.type_addr[p] + i;
                const uint32_t m = poisson_window(idx, net.n_poisson, P.poisson_seed, (double)pop.rate_hz, t0, t1, times);
                for (uint32_t q = 0; q < m; ++q) {
                    ev.emplace_back(times[q], net.base[p] + i);
                    E.sp_time.push_back(times[q]);
                    E.sp_id.push_back(net.base[p] + i);
                }
            }
        }
        std::sort(ev.begin(), ev.end());
        for (const auto& e : ev) {
            const uint32_t T = e.first, src = e.second;
            seg_count.clear();
            for (uint64_t j = net.row_ptr[src]; j < net.row_ptr[src + 1]; ++j) {
                const uint32_t tg = net.tgt[j];
                if (net.kind[tg] == 2) continue;
                if ((flags & 1u) && net.kind[tg] == 1) {
                    const uint32_t g = (tg - nop_base) / 512u;
                    if (g >= seg_count.size()) seg_count.resize(g + 1, 0);
                    if (seg_count[g]++ >= 96u) continue;
                }
                const OrPop& pop = net.pops[net.pop_of[tg]];
                if (T < E.time[tg]) continue;  // dt < 0: refractory
                const double dt = (double)T - (double)E.time[tg];
                float v = (float)((double)E.v[tg] * std::exp(-dt / ((double)pop.tau_m_ms * 1000.0)));
                v = v + net.w[j];
                E.time[tg] = T;
                ++E.delivered;
                if (v > pop.v_th) {
                    E.time[tg] = T + (uint32_t)std::llround((double)pop.t_ref_ms * 1000.0);
                    v = pop.v_reset;
                    E.sp_time.push_back(T);
                    E.sp_id.push_back(tg);
                    E.next.emplace_back(T + W, tg);
                }
                E.v[tg] = v;
            }
        }
        ++E.window;
    }
    return 0;
}

uint64_t oracle_net_event_spike_count(void* h) {
    const Net& net = *static_cast<Net*>(h);
    return net.ev ? net.ev->sp_id.size() : 0;
}

void oracle_net_event_copy(void* h, uint32_t* times, uint32_t* ids, float* v, uint32_t* last_time,
                           uint64_t* delivered) {
    const Net& net = *static_cast<Net*>(h);
    if (!net.ev) return;
    if (times) std::copy(net.ev->sp_time.begin(), net.ev->sp_time.end(), times);
    if (ids) std::copy(net.ev->sp_id.begin(), net.ev->sp_id.end(), ids);
    if (v) std::copy(net.ev->v.begin(), net.ev->v.end(), v);
    if (last_time) std::copy(net.ev->time.begin(), net.ev->time.end(), last_time);
    if (delivered) *delivered = net.ev->delivered;
}

}  // extern "C"
