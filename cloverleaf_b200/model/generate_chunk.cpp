// generate_chunk.cpp -- driver/generate_chunk.h:24: paints the deck's states
// (src/serial/generate_chunk.cpp:31-131) on the device.
#include "generate_chunk.h"
#include "b200_runtime.h"

#include <vector>

void generate_chunk(const int tile, global_variables &globals) {
  std::vector<cb_state> st(globals.config.number_of_states);
  for (int s = 0; s < globals.config.number_of_states; ++s) {
    const state_type &in = globals.config.states[s];
    st[s] = cb_state{in.density, in.energy, in.xvel, in.yvel, (int)in.geometry, in.xmin, in.ymin, in.xmax, in.ymax, in.radius};
  }
  clover::b200_check(cb_generate_chunk(clover::b200_chunk(globals, tile), (int)st.size(), st.data()), "generate_chunk");
}
