// Lifetime hooks for the optional per-context plans (sweep, DSA, solver).
// Each plan's translation unit defines its own; these are the defaults used
// until a plan is built.
#include "ctx.h"

void UboltSweepFree(ubolt_ctx *ctx) { (void)ctx; }
void UboltDsaFree(ubolt_ctx *ctx) { (void)ctx; }
void UboltSolverFree(ubolt_ctx *ctx) { (void)ctx; }
