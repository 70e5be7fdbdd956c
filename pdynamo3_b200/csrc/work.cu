// Algorithmic work of the hot kernels, for roofline reporting, and the stream accessor.
//
// ERI (per Fock build, and per gradient): over the screened quartet list, for every primitive
// quartet that survives the primitive cut, with L_ab = la+lb, L_cd = lc+ld, n_R = (L_ab+L_cd)/2+1
// and n_c the number of Cartesian components,
//   W = n_R [4 n_c + 12 (L_ab+1)(L_cd+1) + 6 (la+1)(lb+1)(L_cd+1) + 6 n_c]
// plus 12 per contracted component integral for the J/K digest.  The gradient uses la+1, lb+1,
// lc+1 in the same formula and 3 times the assembly term, over the quartets the gradient kernels
// evaluate (not one-centre, Schwarz x |Gamma| bound of the last gradient at or above its cut).
// XC (per Fock build): for each grid block with P points and nb functions,
//   rho kernel 2 nb^2 P + 8 nb P, V_xc kernel 4 nb^2 P; bytes = the resident basis values read
//   (4 nb P doubles) by each of the two kernels.
#include <cmath>
#include <cstring>

#include "context.h"

double pdg_grid_work(const pdg_context *ctx, const char *region, double *bytes);

namespace {
constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

double quartet_prim_flops(int la, int lb, int lc, int ld, bool grad) {
    if (grad) { la += 1; lb += 1; lc += 1; }
    const int lab = la + lb, lcd = lc + ld;
    const int nr = (lab + lcd) / 2 + 1;
    const double nc = (double)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    const double assembly = grad ? 3.0 * 4.0 * nc : 4.0 * nc;
    return nr * (assembly + 12.0 * (lab + 1) * (lcd + 1) + 6.0 * (la + 1) * (lb + 1) * (lcd + 1) + 6.0 * nc);
}
}  // namespace

extern "C" int pdg_context_stream(pdg_context *ctx, void **stream) {
    if (!ctx || !stream) return PDG_ERR_ARG;
    *stream = (void *)ctx->stream;
    return PDG_OK;
}

// Algorithmic FLOPs (and bytes where meaningful) of one call of a region ("eri_jk", "eri_grad",
// "xc_rho", "xc_vxc") for the current geometry and screening.
extern "C" int pdg_work_estimate(pdg_context *ctx, const char *region, double *flops, double *bytes,
                                 long long *quartets) {
    if (!ctx || !region || !flops) { pdg_set_error("pdg_work_estimate: invalid argument"); return PDG_ERR_ARG; }
    *flops = 0.0;
    if (bytes) *bytes = 0.0;
    if (quartets) *quartets = 0;
    const bool grad = std::strcmp(region, "eri_grad") == 0;
    if (grad || std::strcmp(region, "eri_jk") == 0) {
        PDG_CHECK(pdg_ensure_pairs(ctx));
        PDG_CHECK(pdg_build_blocks(ctx, ctx->schwarz_cut));
        // The gradient kernels skip one-centre quartets and those whose Schwarz x |Gamma| bound is
        // below the cut of the last gradient: count only the quartets they evaluate, by the same
        // rule on the density maxima that gradient used.
        const int ns = (int)ctx->shells.size();
        const bool gscreen = grad && ctx->grad_valid;
        std::vector<double> m;
        std::vector<int> shA[PDG_NPAIRCLASS], shB[PDG_NPAIRCLASS];
        if (gscreen) {
            const double *d_m = (const double *)pdg_pool(ctx, "grad_dmax", (size_t)ns * ns * sizeof(double));
            if (!d_m) { pdg_set_error("pdg_work_estimate: device buffer allocation failed"); return PDG_ERR_ALLOC; }
            m.resize((size_t)ns * ns);
            PDG_CUDA(cudaMemcpyAsync(m.data(), d_m, m.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            for (int c = 0; c < PDG_NPAIRCLASS; ++c) {
                const int np = ctx->pairs[c].n;
                shA[c].resize(np);
                shB[c].resize(np);
                if (np == 0) continue;
                PDG_CUDA(cudaMemcpyAsync(shA[c].data(), ctx->pairs[c].shA, np * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
                PDG_CUDA(cudaMemcpyAsync(shB[c].data(), ctx->pairs[c].shB, np * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            }
            PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        const double gcx = std::fabs(ctx->grad_cx), gj = ctx->grad_doJ ? 4.0 : 0.0;
        auto grad_evaluated = [&](int cb, int ib, int ck, int ik) {
            const int A = shA[cb][ib], B = shB[cb][ib], C = shA[ck][ik], D = shB[ck][ik];
            const int at = ctx->shells[A].atom;
            if (ctx->shells[B].atom == at && ctx->shells[C].atom == at && ctx->shells[D].atom == at) return false;
            const double gam = gj * m[(size_t)A * ns + B] * m[(size_t)C * ns + D] +
                               gcx * (m[(size_t)A * ns + C] * m[(size_t)B * ns + D] + m[(size_t)A * ns + D] * m[(size_t)B * ns + C]);
            return ctx->hostQ[cb][ib] * ctx->hostQ[ck][ik] * gam >= ctx->grad_gcut;
        };
        double w = 0.0;
        long long nq = 0;
        for (const auto &b : ctx->blocks) {
            const int la = PLA[b.cb], lb = PLB[b.cb], lc = PLA[b.ck], ld = PLB[b.ck];
            const double fq = quartet_prim_flops(la, lb, lc, ld, grad);
            const double digest = 12.0 * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
            const auto &Qb = ctx->hostQ[b.cb];
            for (int k = 0; k < b.nsub; ++k) {
                const auto &sb = b.sub[k];
                for (size_t ib = 0; ib < Qb.size(); ++ib) {
                    // the same count rule as the work lists
                    const long long cnt = pdg_ket_count(ctx, b.cb, b.ck, (int)ib, sb.k0, sb.nk, ctx->schwarz_cut);
                    const int pb0 = ctx->hostPoff[b.cb][ib], npb = ctx->hostNp[b.cb][ib];
                    for (long long ik = sb.k0; ik < sb.k0 + cnt; ++ik) {
                        if (gscreen && !grad_evaluated(b.cb, (int)ib, b.ck, (int)ik)) continue;
                        const int pk0 = ctx->hostPoff[b.ck][ik], npk = ctx->hostNp[b.ck][ik];
                        long long nprim = 0;
                        for (int x = 0; x < npb; ++x) {
                            const double ab = ctx->hostArg[pb0 + x];
                            for (int y = 0; y < npk; ++y)
                                if (ab + ctx->hostArg[pk0 + y] <= PDG_PRIMITIVE_CUT) ++nprim;
                        }
                        w += nprim * fq + (grad ? 0.0 : digest);
                        ++nq;
                    }
                }
            }
        }
        *flops = w;
        if (quartets) *quartets = nq;
        return PDG_OK;
    }
    if (std::strcmp(region, "eri_jk_fp32") == 0) {
        // shell quartets evaluated in FP32 since the context's first mixed-precision build
        unsigned long long c = 0;
        if (ctx->d_count32) {
            PDG_CUDA(cudaMemcpyAsync(&c, ctx->d_count32, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
            PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        if (quartets) *quartets = (long long)c;
        return PDG_OK;
    }
    if (std::strcmp(region, "xc_rho") == 0 || std::strcmp(region, "xc_vxc") == 0) {
        double by = 0.0;
        *flops = pdg_grid_work(ctx, region, &by);
        if (bytes) *bytes = by;
        return PDG_OK;
    }
    pdg_set_error("pdg_work_estimate: unknown region '%s'", region);
    return PDG_ERR_ARG;
}
