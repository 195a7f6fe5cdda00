// The complex128 kernels of the QFT / Walsh pass (qft_pass.cu), in a unit of
// their own so that the two precisions compile in parallel.
#define TMFQS_QFT_UNIT_C128
#include "qft_pass.cu"
