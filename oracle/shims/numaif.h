/* Declaration-only stand-in for libnuma's <numaif.h> (absent in this image).
 * The reference's HostMem (core/mem.hpp:258,301) queries the NUMA node of a
 * pinned buffer; the oracle harness never instantiates HostMem, so only the
 * declaration is needed for the header to parse. */
#pragma once
#define MPOL_F_NODE (1 << 0)
#define MPOL_F_ADDR (1 << 1)
#ifdef __cplusplus
extern "C" {
#endif
long get_mempolicy(int* mode, unsigned long* nodemask, unsigned long maxnode, void* addr, unsigned flags);
#ifdef __cplusplus
}
#endif
