/* The reference's Poisson-generator, random-number and connectivity kernels
 * (include/naer/kernels/input_neuron_group.cl, random.cl, network.cl),
 * compiled unchanged from the reference's own sources by oracle/Makefile
 * (target `ref`) and run on the host under clshim.h: the checker the
 * oracle's restatement is compared with.  Test infrastructure only. */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "clshim.h"

#define NAER_NUM_GROUPS 64     /* destination groups of one connectivity run */
#define NAER_NUM_NEURONS 8192  /* source rows of one connectivity run */
#define CLSHIM_SPIKE_CAPACITY 65536
#include "input_neuron_group.cl"
#include "network.cl"

__thread struct clshim_item clshim_self;

static pthread_barrier_t g_barrier;
static size_t g_barrier_n;

void barrier(int flags) {
    (void)flags;
    if (g_barrier_n > 1) pthread_barrier_wait(&g_barrier);
}

struct clshim_thread {
    struct clshim_item id;
    void (*item)(void*);
    void* arg;
};

static void* clshim_thread_main(void* p) {
    struct clshim_thread* t = (struct clshim_thread*)p;
    clshim_self = t->id;
    t->item(t->arg);
    return NULL;
}

void clshim_run(size_t groups, size_t local_size, void (*item)(void*), void* arg) {
    pthread_t* th = (pthread_t*)malloc(local_size * sizeof(pthread_t));
    struct clshim_thread* ta = (struct clshim_thread*)malloc(local_size * sizeof(struct clshim_thread));
    g_barrier_n = local_size;
    if (local_size > 1) pthread_barrier_init(&g_barrier, NULL, (unsigned)local_size);
    for (size_t g = 0; g < groups; ++g) {
        for (size_t l = 0; l < local_size; ++l) {
            ta[l].id.global_id = g * local_size + l;
            ta[l].id.group_id = g;
            ta[l].id.local_id = l;
            ta[l].id.local_size = local_size;
            ta[l].item = item;
            ta[l].arg = arg;
            if (local_size == 1) {
                clshim_thread_main(&ta[l]);
            } else if (pthread_create(&th[l], NULL, clshim_thread_main, &ta[l]) != 0) {
                fprintf(stderr, "clshim: cannot start work-item thread %zu of %zu\n", l, local_size);
                abort();  /* the group's barrier could never complete */
            }
        }
        if (local_size > 1)
            for (size_t l = 0; l < local_size; ++l) pthread_join(th[l], NULL);
    }
    if (local_size > 1) pthread_barrier_destroy(&g_barrier);
    free(ta);
    free(th);
}

/* ------------------------------------------------------------------------ */

void ref_philox4x32(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]) {
    philox4x32_ctr_t x = {{c[0], c[1], c[2], c[3]}};
    philox4x32_key_t y = {{k[0], k[1]}};
    x = philox4x32(x, y);
    memcpy(out, x.v, sizeof(x.v));
}

/* random.cl's uniform_rand / exprnd on the work-item with global id gid */
double ref_uniform_rand(uint32_t gid, uint32_t seed, uint32_t iteration) {
    clshim_self.global_id = gid;
    return uniform_rand(seed, iteration);
}

double ref_exprnd(uint32_t gid, double rate, uint32_t seed, uint32_t iteration) {
    clshim_self.global_id = gid;
    return exprnd(rate, seed, iteration);
}

/* simulate_poisson_neurons (input_neuron_group.cl:6-45, 20 Hz) for one
 * window [prev_time, next_time): `total` generators in groups of
 * `capacity`, work-groups of `local_size`.  Writes up to `cap` spikes
 * (time, address) and returns how many the kernel emitted. */
struct poisson_args {
    spike_buffer* out;
    uint* sizes;
    uint total, capacity, seed, t0, t1;
};

static void poisson_item(void* p) {
    struct poisson_args* a = (struct poisson_args*)p;
    simulate_poisson_neurons(a->out, a->sizes, a->total, a->capacity, 0u, 0u, a->seed, a->t0, a->t1);
}

uint32_t ref_poisson_neurons(uint32_t total, uint32_t capacity, uint32_t local_size, uint32_t seed,
                             uint32_t prev_time, uint32_t next_time, uint32_t* times, uint32_t* addresses,
                             uint32_t cap) {
    const uint32_t groups = (total + capacity - 1) / capacity;
    struct poisson_args a;
    a.out = (spike_buffer*)calloc(groups, sizeof(spike_buffer));
    a.sizes = (uint*)calloc(groups, sizeof(uint));
    a.total = total;
    a.capacity = capacity;
    a.seed = seed;
    a.t0 = prev_time;
    a.t1 = next_time;
    clshim_run(groups, local_size, poisson_item, &a);
    uint32_t n = 0;
    for (uint32_t g = 0; g < groups; ++g)
        for (uint32_t k = 0; k < a.sizes[g]; ++k, ++n)
            if (n < cap) {
                times[n] = a.out[g].times[k];
                addresses[n] = a.out[g].addresses[k];
            }
    free(a.sizes);
    free(a.out);
    return n;
}

/* count_connections, integrate_connections and generate_connections
 * (network.cl:14-107) for one connection from a population of src_size
 * neurons (one work-group of 32 per source, as the reference launches it)
 * onto a population of dst_size neurons in groups of group_capacity.
 * Writes up to `cap` synapses as (source, destination, weight) and returns
 * how many the kernels generated; ~0 when the sizes exceed this build's
 * NAER_NUM_NEURONS / NAER_NUM_GROUPS. */
struct net_args {
    uint (*offsets)[NAER_NUM_GROUPS + 1];
    float* weights;
    ushort* local_addresses;
    uint seed, dst_size, group_capacity;
    double p;
    float w, wmin, wmax;
};

static void count_item(void* p) {
    struct net_args* a = (struct net_args*)p;
    count_connections(a->offsets, 0u, a->seed, a->dst_size, 0u, 0u, 0u, a->group_capacity, a->p);
}

static void integrate_item(void* p) {
    struct net_args* a = (struct net_args*)p;
    integrate_connections(a->offsets);
}

static void generate_item(void* p) {
    struct net_args* a = (struct net_args*)p;
    generate_connections(a->offsets, a->weights, a->local_addresses, 0u, a->seed, a->dst_size, 0u, 0u, 0u,
                         a->group_capacity, a->p, a->w, a->wmin, a->wmax);
}

uint64_t ref_bernoulli(uint32_t src_size, uint32_t dst_size, uint32_t group_capacity, uint32_t seed, double p,
                       float w, float wmin, float wmax, uint32_t* src_out, uint32_t* dst_out, float* w_out,
                       uint64_t cap) {
    const uint32_t dst_groups = (dst_size + group_capacity - 1) / group_capacity;
    if (src_size > NAER_NUM_NEURONS || dst_groups > NAER_NUM_GROUPS) return ~(uint64_t)0;
    struct net_args a;
    a.offsets = (uint(*)[NAER_NUM_GROUPS + 1])calloc((size_t)NAER_NUM_NEURONS * (NAER_NUM_GROUPS + 1), sizeof(uint));
    a.seed = seed;
    a.dst_size = dst_size;
    a.group_capacity = group_capacity;
    a.p = p;
    a.w = w;
    a.wmin = wmin;
    a.wmax = wmax;
    clshim_run(src_size, 32, count_item, &a);
    uint* counts = (uint*)malloc((size_t)NAER_NUM_NEURONS * (NAER_NUM_GROUPS + 1) * sizeof(uint));
    memcpy(counts, a.offsets, (size_t)NAER_NUM_NEURONS * (NAER_NUM_GROUPS + 1) * sizeof(uint));
    uint64_t total = 0;
    for (size_t i = 0; i < (size_t)NAER_NUM_NEURONS * (NAER_NUM_GROUPS + 1); ++i) total += counts[i];
    clshim_run(1, 1, integrate_item, &a);
    a.weights = (float*)calloc(total + 1, sizeof(float));
    a.local_addresses = (ushort*)calloc(total + 1, sizeof(ushort));
    clshim_run(src_size, 32, generate_item, &a);
    uint64_t n = 0;
    for (uint32_t s = 0; s < src_size; ++s)
        for (uint32_t g = 0; g < dst_groups; ++g) {
            const uint first = a.offsets[s][g];
            const uint c = counts[(size_t)s * (NAER_NUM_GROUPS + 1) + g];
            for (uint e = first; e < first + c; ++e, ++n)
                if (n < cap) {
                    src_out[n] = s;
                    dst_out[n] = g * group_capacity + a.local_addresses[e];
                    w_out[n] = a.weights[e];
                }
        }
    free(a.local_addresses);
    free(a.weights);
    free(counts);
    free(a.offsets);
    return n;
}
