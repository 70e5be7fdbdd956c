// DFT grid integrator (placeholder until the grid kernels land).
#include "context.h"

bool pdg_dft_active(const pdg_context *ctx) { return ctx->xc != nullptr; }
double pdg_dft_exchange_scaling(const pdg_context *) { return 1.0; }
double pdg_dft_last_vxc_trace(const pdg_context *) { return 0.0; }
int pdg_dft_fock_device(pdg_context *, double *, double *, double *) { return PDG_ERR_UNSUPPORTED; }
int pdg_dft_grad_device(pdg_context *, double *) { return PDG_ERR_UNSUPPORTED; }
void pdg_free_dft(pdg_context *) {}

extern "C" int pdg_set_functional(pdg_context *ctx, const char *name, double *cx) {
    if (!ctx || !name) return PDG_ERR_ARG;
    if (cx) *cx = 1.0;
    return PDG_ERR_UNSUPPORTED;
}
extern "C" int pdg_grid_build(pdg_context *, int, int, int, long long *) { return PDG_ERR_UNSUPPORTED; }
extern "C" int pdg_fock_quadrature(pdg_context *, const double *, double *, double *, double *) { return PDG_ERR_UNSUPPORTED; }
extern "C" int pdg_gradients_quadrature(pdg_context *, const double *, double *) { return PDG_ERR_UNSUPPORTED; }
