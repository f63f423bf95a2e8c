/* The reference includes "spikes.cl", which its snapshot does not contain.
 * Its kernels use `spike_buffer` with the fields of the spike record in
 * naer_types.h; this stand-in declares it with that header's macro and a
 * capacity the including translation unit chooses. */
#ifndef CLSHIM_SPIKES_CL
#define CLSHIM_SPIKES_CL
#include "naer_types.h"
#ifndef CLSHIM_SPIKE_CAPACITY
#define CLSHIM_SPIKE_CAPACITY 4096
#endif
DECLARE_SPIKE_BUFFER(CLSHIM_SPIKE_CAPACITY, spike_buffer);
#endif
