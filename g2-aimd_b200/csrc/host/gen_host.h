// gen_host.h - host pieces of the seeded generators shared with the device
// generator (csrc/gen.cu); internal to libg2aimd.so.
#pragma once

#include <cstdint>
#include <vector>

namespace g2host {
// Edges (src << 32 | dst) of `count` cliques of smin..smax vertices on disjoint
// random vertex sets, exactly as g2_gen_er / g2_gen_rmat plant them.
int planted_edges(uint64_t n, uint32_t count, uint32_t smin, uint32_t smax, uint64_t seed,
                  std::vector<uint64_t> &edges);
}  // namespace g2host
