// design_inst_col_fourier.cu -- far-field (fourierCgh) column passes, every length
// and shape variant.
#define DOE_DESIGN_INSTANTIATE
#include "design_ops.cuh"

namespace doe {
DOE_DESIGN_COL_INST(ColFourier<true>)
DOE_DESIGN_COL_INST(ColFourier<false>)
}  // namespace doe
