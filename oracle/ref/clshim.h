/* Host shim under which the reference's OpenCL C kernels compile as C11
 * (test infrastructure: the checker's reference build, never the product).
 *
 * A kernel runs over an NDRange as in OpenCL: every work-item of a
 * work-group is a host thread, work-groups run one after another, `local`
 * variables of a kernel are statics shared by the group's threads, and
 * barrier() waits for the whole group.  The work-item functions read the
 * calling thread's ids.  A translation unit whose kernels use `local` only
 * as a pointer qualifier defines CLSHIM_LOCAL_AS_QUALIFIER before including
 * this header. */
#ifndef CLSHIM_H
#define CLSHIM_H

#include <limits.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <sys/types.h>

typedef unsigned int uint;
typedef unsigned short ushort;
typedef unsigned long ulong;
typedef unsigned char uchar;
typedef struct {
    int x, y, z, w;
} int4;

#define kernel
#define __kernel
#define global
#define __global
#define constant const
#ifdef CLSHIM_LOCAL_AS_QUALIFIER
#define local
#else
#define local static
#endif

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

struct clshim_item {
    size_t global_id, group_id, local_id, local_size;
};
extern __thread struct clshim_item clshim_self;

static inline size_t get_global_id(uint d) { return d == 0 ? clshim_self.global_id : 0; }
static inline size_t get_group_id(uint d) { return d == 0 ? clshim_self.group_id : 0; }
static inline size_t get_local_id(uint d) { return d == 0 ? clshim_self.local_id : 0; }
static inline size_t get_local_size(uint d) { return d == 0 ? clshim_self.local_size : 1; }

void barrier(int flags);

static inline uint atomic_inc(volatile uint* p) { return __atomic_fetch_add(p, 1u, __ATOMIC_SEQ_CST); }
static inline uint atomic_add(volatile uint* p, uint v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }

#define min(a, b) ((a) < (b) ? (a) : (b))
#define max(a, b) ((a) > (b) ? (a) : (b))

/* Runs item(arg) on every work-item of an NDRange of `groups` work-groups of
 * `local_size` work-items (dimension 0). */
void clshim_run(size_t groups, size_t local_size, void (*item)(void*), void* arg);

#endif
