// design_inst_update.cu -- DOE-plane update row passes that chain into the next
// forward transform, every length and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_ROW_INST(RowDoeUpdate<true, false, false>)
DOE_DESIGN_ROW_INST(RowDoeUpdate<true, true, false>)
DOE_DESIGN_ROW_INST(RowDoeUpdate<true, true, true>)
}  // namespace doe
