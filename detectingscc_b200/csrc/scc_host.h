// Host-only declarations shared by the C++ translation units.
#pragma once
#include <cstdint>

#include "../../include/scc_b200.h"

int scc_build_csr(uint32_t V, uint64_t E, const uint32_t *src, const uint32_t *dst, scc_host_graph *g);
