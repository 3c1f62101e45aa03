// tcgen05 tensor-core r12 contraction (sm_100a): placeholder until the kernel lands.
#include "kernels.cuh"

namespace tcscf {

bool tensorPathAvailable(Contraction const &, int, std::string * why)
{
  if (why) *why = "tensor-core path not built";
  return false;
}

int contractTensor(tcscf_ctx * ctx, Contraction const &, int)
{
  return fail(ctx, TCSCF_ERR_UNSUPPORTED, "tensor-core path not built");
}

}  // namespace tcscf
