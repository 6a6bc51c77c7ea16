// setup_from: the g3d structs of a run from the reference's Config (src/sim.hpp:36-187), the mapping of the deck keys
// (docs/input_deck.md of the reference) onto the C-ABI. Compiled against the reference's own headers.
#pragma once
#include "g3d_simulation.hpp"

struct Config;

namespace g3dshim {
// Throws std::runtime_error naming the first key or feature of the Config that libg3d does not run.
Setup setup_from(const Config& c);
}  // namespace g3dshim
