/* Hardware constants for building the reference's execute() on this host:
 * thread count and cache sizes come from -D flags (the reference hard-codes
 * a 16-core / 32-thread Ryzen in its own platform/hardware.h).
 * TEST INFRASTRUCTURE. */
#pragma once
#ifndef SPC__THREAD_COUNT
#define SPC__THREAD_COUNT 32
#endif
#ifndef SPC__CORE_COUNT
#define SPC__CORE_COUNT SPC__THREAD_COUNT
#endif
#ifndef SPC__LEVEL1_DCACHE_SIZE
#define SPC__LEVEL1_DCACHE_SIZE 49152
#endif
#ifndef SPC__LEVEL2_CACHE_SIZE
#define SPC__LEVEL2_CACHE_SIZE 2097152
#endif
#ifndef SPC__LEVEL3_CACHE_SIZE
#define SPC__LEVEL3_CACHE_SIZE 134217728
#endif
#ifndef SPC__LEVEL1_DCACHE_LINESIZE
#define SPC__LEVEL1_DCACHE_LINESIZE 64
#endif
#ifndef SPC__NUMA_NODE_DRAM_MB
#define SPC__NUMA_NODE_DRAM_MB 24576
#endif
