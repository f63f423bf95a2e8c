/* The reference's neuron update, neuron_dynamics (include/naer/kernels/
 * lif.cl:15-34), compiled unchanged from its own source by oracle/Makefile
 * (target `ref`): one neuron driven by a sequence of input events.  Test
 * infrastructure only. */
#define CLSHIM_LOCAL_AS_QUALIFIER
#include "clshim.h"

#define NAER_GROUP_SIZE 512
#include "lif.cl"

/* Applies events (times[i] in us, weights[i]) in order to neuron 0 of a
 * zeroed group; fired[i] = 1 where the event made it spike.  Returns the
 * final potential and last-event time through v and t_last. */
void ref_neuron_dynamics_run(const uint32_t* times, const float* weights, uint32_t n, float* v, uint32_t* t_last,
                             uint8_t* fired) {
    static neuron_group g;
    g.potential[0] = 0.0f;
    g.time[0] = 0u;
    for (uint32_t i = 0; i < n; ++i) {
        spike s;
        synapse y;
        s.times[0] = times[i];
        y.weights[0] = weights[i];
        fired[i] = neuron_dynamics(&g, 0u, &s, &y) ? 1u : 0u;
    }
    *v = g.potential[0];
    *t_last = g.time[0];
}
