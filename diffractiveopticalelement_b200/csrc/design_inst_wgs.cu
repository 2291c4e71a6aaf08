// design_inst_wgs.cu -- target-plane row passes of image-plane
// weightedGerchbergSaxton, every length and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_ROW_INST(RowWgsTarget<false, false>)
DOE_DESIGN_ROW_INST(RowWgsTarget<false, true>)
DOE_DESIGN_ROW_INST(RowWgsTarget<true, false>)
DOE_DESIGN_ROW_INST(RowWgsTarget<true, true>)
DOE_DESIGN_ROW_INST(RowWgsConstrain)
}  // namespace doe
