// design_inst_doe.cu -- first forward and last DOE-plane row passes, every length
// and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_ROW_INST(RowDoeFwd<false>)
DOE_DESIGN_ROW_INST(RowDoeFwd<true>)
DOE_DESIGN_ROW_INST(RowDoeUpdate<false, false, false>)
DOE_DESIGN_ROW_INST(RowDoeUpdate<false, true, false>)
DOE_DESIGN_ROW_INST(RowDoeUpdate<false, true, true>)
}  // namespace doe
