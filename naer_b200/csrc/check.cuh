// Bounds checks of the NAER_CHECKED build (libnaer_b200_checked.so).
//
// Every global access the step kernels make at a computed index is guarded
// by NAER_IN_BOUNDS(ctl, index, bound, code): in the checked build an index
// outside its buffer is not accessed; the first one is recorded in the
// control block (Ctl::chk_code, chk_index) and reported by
// naer_net_check_report.  The normal build compiles the guards away.  This
// is the project's own bounds check for a pool where no sanitizer runs.
#pragma once
#include "engine_types.cuh"

namespace naer {

enum CheckCode : uint32_t {
    kChkNone = 0,
    kChkSynapse = 1,    // synapse array offset (target / weight / delay)
    kChkRing = 2,       // ring cell
    kChkQueue = 3,      // source of a queued spike
    kChkState = 5,      // neuron state of a LIF chunk
    kChkDrive = 6,      // Poisson-count slot
    kChkEventList = 8,  // deterministic event list (synapse slot)
};

#ifdef NAER_CHECKED
__device__ __forceinline__ bool naer_in_bounds(Ctl* ctl, unsigned long long idx, unsigned long long bound,
                                               uint32_t code) {
    if (idx < bound) return true;
    if (atomicCAS(&ctl->chk_code, 0u, code) == 0u) ctl->chk_index = idx;
    return false;
}
#define NAER_IN_BOUNDS(ctl, idx, bound, code) \
    ::naer::naer_in_bounds((ctl), (unsigned long long)(idx), (unsigned long long)(bound), (code))
#else
#define NAER_IN_BOUNDS(ctl, idx, bound, code) true
#endif

}  // namespace naer
