// tcb_unit.cu — standalone batched kernels (filled in below).
#include "tcb_launch.h"
#include "tcb_resid.cuh"
namespace tcb {
cudaError_t init_unit_tables() { return upload_dct_tables(); }
}
