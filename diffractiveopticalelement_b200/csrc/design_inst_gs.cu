// design_inst_gs.cu -- target-plane row passes of gerchbergSaxton and of the
// multi-plane loop, every length and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_ROW_INST(RowGsTarget<false, false>)
DOE_DESIGN_ROW_INST(RowGsTarget<false, true>)
DOE_DESIGN_ROW_INST(RowGsTarget<true, false>)
}  // namespace doe
