// Superposition-of-atomic-densities (SAD) initial density.
//
// For every element present, a Hartree-Fock calculation of the isolated atom in the molecule's
// own basis is run once per basis upload on this device, with spherically averaged fractional
// occupations (the open p shell shared equally by its three orbitals), and its density is kept.
// The molecular guess is the block-diagonal sum of the atomic densities.  The reference starts
// from a uniform diagonal density instead (pMolecule/QCModel/QCOnePDM.py:51-67); the guess
// changes the number of SCF cycles only, not the converged energy or gradient.
#include <cmath>
#include <vector>

#include <map>
#include <mutex>
#include <string>

#include "context.h"

extern "C" int pdg_context_create(int device, pdg_context **out);
extern "C" int pdg_context_destroy(pdg_context *ctx);
extern "C" int pdg_basis_upload(pdg_context *ctx, int n_atoms, const double *Z, int n_shells, const int *shell_atom,
                                const int *l_low, const int *l_high, const int *nprim, const double *exponents,
                                const double *coefficients, int normalized, int spherical);
extern "C" int pdg_geometry_set(pdg_context *ctx, const double *xyz);
extern "C" int pdg_scf_run(pdg_context *ctx, const pdg_scf_options *opt, double *density, pdg_scf_result *res);

namespace {

// Ground-state configuration averaged over the open shell, orbitals in the order 1s 2s 2p(3) 3s 3p(3).
bool atomic_occupations(int z, std::vector<double> &occ) {
    occ.clear();
    if (z < 1 || z > 18) return false;
    const int caps[] = {2, 2, 6, 2, 6};  // 1s 2s 2p 3s 3p
    const int orbs[] = {1, 1, 3, 1, 3};
    int left = z;
    for (int s = 0; s < 5 && left > 0; ++s) {
        const int e = left < caps[s] ? left : caps[s];
        for (int k = 0; k < orbs[s]; ++k) occ.push_back((double)e / orbs[s]);
        left -= e;
    }
    return true;
}

int atomic_density(pdg_context *ctx, int atom, std::vector<double> &packed) {
    const auto &ra = ctx->raw_atom[atom];
    const int z = (int)std::lround(ctx->Z[atom]);
    std::vector<double> occ;
    if (!atomic_occupations(z, occ) || ra.np.empty()) return PDG_ERR_UNSUPPORTED;
    pdg_context *sub = nullptr;
    PDG_CHECK(pdg_context_create(ctx->device, &sub));
    const int ns = (int)ra.np.size();
    std::vector<int> sa(ns, 0);
    const double zz = ctx->Z[atom];
    int st = pdg_basis_upload(sub, 1, &zz, ns, sa.data(), ra.llo.data(), ra.lhi.data(), ra.np.data(), ra.ex.data(),
                              ra.co.data(), ctx->raw_normalized, ctx->spherical);
    const double origin[3] = {0.0, 0.0, 0.0};
    if (st == PDG_OK) st = pdg_geometry_set(sub, origin);
    if (st == PDG_OK) {
        sub->occ = occ;
        sub->guess_sad = 0;
        pdg_scf_options o{};
        o.density_tolerance = 1.0e-6;
        o.energy_tolerance = 1.0e-6;
        o.maximum_iterations = 60;
        o.maximum_history = 8;
        o.use_guess = 0;
        o.total_charge = 0.0;
        pdg_scf_result r{};
        packed.assign((size_t)sub->nbf_out * (sub->nbf_out + 1) / 2, 0.0);
        st = pdg_scf_run(sub, &o, packed.data(), &r);
        if (st == PDG_ERR_NOCONV) st = PDG_OK;  // an unconverged atom is still a usable guess
    }
    pdg_context_destroy(sub);
    return st;
}

// Bytes that identify an atom's guess density: nuclear charge, normalisation and spherical flags,
// and its shells as uploaded.
std::string atom_signature(const pdg_context *ctx, int atom) {
    const auto &ra = ctx->raw_atom[atom];
    std::string k;
    auto put = [&k](const void *p, size_t n) { k.append(reinterpret_cast<const char *>(p), n); };
    const double z = ctx->Z[atom];
    put(&z, sizeof z);
    put(&ctx->raw_normalized, sizeof ctx->raw_normalized);
    put(&ctx->spherical, sizeof ctx->spherical);
    const size_t ns = ra.np.size();
    put(&ns, sizeof ns);
    put(ra.llo.data(), ra.llo.size() * sizeof(int));
    put(ra.lhi.data(), ra.lhi.size() * sizeof(int));
    put(ra.np.data(), ra.np.size() * sizeof(int));
    put(ra.ex.data(), ra.ex.size() * sizeof(double));
    put(ra.co.data(), ra.co.size() * sizeof(double));
    return k;
}

std::mutex g_sad_mutex;
std::map<std::string, std::vector<double>> g_sad_cache;

}  // namespace

int pdg_sad_density(pdg_context *ctx, std::vector<double> &full) {
    const int m = ctx->nbf_out;
    // output-basis offset and size of each atom's block (functions are ordered by atom)
    std::vector<int> first(ctx->natom, -1), count(ctx->natom, 0);
    {
        int off = 0;
        for (const auto &h : ctx->shells) {
            const int nf = ctx->spherical ? 2 * h.l + 1 : ncart(h.l);
            if (first[h.atom] < 0) first[h.atom] = off;
            count[h.atom] += nf;
            off += nf;
        }
    }
    for (int a = 0; a < ctx->natom; ++a) {
        const int z = (int)std::lround(ctx->Z[a]);
        if (ctx->sad.count(z)) continue;
        // the process-wide cache: an element with the same shells (exponents, coefficients,
        // normalisation, spherical flag) has the same atomic density in every context
        const std::string key = atom_signature(ctx, a);
        {
            std::lock_guard<std::mutex> lock(g_sad_mutex);
            auto it = g_sad_cache.find(key);
            if (it != g_sad_cache.end()) { ctx->sad[z] = it->second; continue; }
        }
        std::vector<double> pk;
        const int st = atomic_density(ctx, a, pk);
        if (st != PDG_OK) return st;
        ctx->sad[z] = pk;
        std::lock_guard<std::mutex> lock(g_sad_mutex);
        g_sad_cache.emplace(key, pk);
    }
    cudaSetDevice(ctx->device);
    full.assign((size_t)m * m, 0.0);
    for (int a = 0; a < ctx->natom; ++a) {
        const auto &pk = ctx->sad[(int)std::lround(ctx->Z[a])];
        const int n = count[a], o = first[a];
        if ((size_t)n * (n + 1) / 2 != pk.size()) return PDG_ERR_STATE;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= i; ++j) {
                const double v = pk[(size_t)i * (i + 1) / 2 + j];
                full[(size_t)(o + i) * m + o + j] = v;
                full[(size_t)(o + j) * m + o + i] = v;
            }
    }
    return PDG_OK;
}
