// Defaults for the optional DSA stage until its plan is built (dsa.cu
// replaces these when present).
#include "ctx.h"

void UboltDsaFree(ubolt_ctx *ctx) { (void)ctx; }

namespace ubolt {
template <typename T>
int DsaCorrect(ubolt_ctx *ctx, const T *r, T *y, T *tmp, void *stream)
{
   (void)ctx; (void)r; (void)y; (void)tmp; (void)stream;
   return SetError(UBOLT_ERR_STATE, "no DSA stage in this build");
}
template int DsaCorrect<double>(ubolt_ctx *, const double *, double *, double *, void *);
template int DsaCorrect<float>(ubolt_ctx *, const float *, float *, float *, void *);
}  // namespace ubolt
