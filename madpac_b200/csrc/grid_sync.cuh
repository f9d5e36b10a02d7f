// Grid-wide barrier with a bounded wait, for cooperative launches (all CTAs co-resident).
// bar[0] counts arrivals, bar[1] is the generation. A wait that runs out of its time limit sets
// the timeout status and returns false; the caller then skips the rest of the launch and the host
// resets bar[] after reading the status.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "md_internal.h"

namespace mdgpu {

__device__ __forceinline__ uint64_t global_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ unsigned load_acquire(const unsigned* p) {
	unsigned v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

// Grid-wide barrier with a bounded wait. Returns false (and sets the timeout status) when the wait
// ran out; the caller then skips the rest of the launch.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, int64_t timeout_ns, int* s_flag) {
	__syncthreads();
	if (threadIdx.x == 0) {
		const unsigned gen = load_acquire(bar + 1);
		__threadfence();
		const unsigned arrived = atomicAdd(bar, 1u);
		if (arrived == gridDim.x - 1) {
			atomicExch(bar, 0u);
			__threadfence();
			atomicAdd(bar + 1, 1u);
		} else {
			const uint64_t t0 = global_ns();
			while (load_acquire(bar + 1) == gen) {
				__nanosleep(100);
				if ((int64_t) (global_ns() - t0) > timeout_ns) {
					atomicOr(status, kStatusTimeout);
					*s_flag = 1;
					break;
				}
			}
		}
		__threadfence();
	}
	__syncthreads();
	return *s_flag == 0;
}

}  // namespace mdgpu
