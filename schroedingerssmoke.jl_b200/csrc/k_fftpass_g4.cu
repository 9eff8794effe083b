// Grouped-tile (G = 4) instantiations of the FFT pass launchers.
#include "k_fftpass_impl.cuh"

namespace isf {

#define ISF_INST(NN) ISF_GROUPED_DECLS(, NN, 4)
ISF_GROUPED_SIZES(ISF_INST)
#undef ISF_INST

}  // namespace isf
