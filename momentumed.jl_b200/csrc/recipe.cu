// Two-body amplitudes regenerated on the device for twisted-boundary sweeps.
//
// With momentum coordinates, ED_scatterlist_twobody (MomentumED/src/preparation/scat_list.jl:
// 442-497) evaluates H_two at k/Gk + kshift/Gk of each conserved component (scat_list.jl:5-50),
// so every point of a twisted-boundary sweep (the Wilson loops of many-body Chern numbers)
// rebuilds the whole term list on the host.  The STRUCTURE of the list (which (out, in) masks
// appear, with which normal-ordering signs and which raw contributions merge into each term)
// does not depend on kshift; only the amplitudes do.  The host describes the structure once
// (momed_set_twobody_recipe: per upper term its raw contributions (kf1, kf2, ki2, ki1,
// cf1, cf2, ci2, ci1, sign, conj / real part) in the order the reference's sort_merge sums
// them); momed_set_kshift then evaluates a built-in interaction on the device for all of them,
// sums each upper term, and writes the Hermitian-completed amplitudes (FP64 and the FP32 copy)
// straight into the handle's term slots.  No host round trip per sweep point.
//
// Built-in interaction (MOMED_RECIPE_LANDAU_COULOMB): the screened Coulomb interaction projected
// to the lowest Landau level with magnetic-translation phases, the H_two of the reference's own
// test (MomentumED/test/example1_FQH_Laughlin.jl:20-89), on momentum coordinates:
//   V = sum_{g1, g2, |g1|,|g2|,|g1-g2| <= nshell} sgn * exp(i pi 2 phi) * VFF(q + g)
//   VFF(q) = W0 / |q l| tanh(|q l| D) exp(-|q l|^2 / 2)   (W0 D at q = 0)
// with the reciprocal metric of angle theta between the two reciprocal vectors.  params:
// [Gl (magnetic length scale), D (screening / l), W0, theta, nshell].  Components are ignored
// (as by that H_two: one component).  The device evaluates it in FP64 with CUDA's sincospi,
// tanh and exp, so amplitudes agree with the host builder to ~1e-15 relative, not bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "momed_internal.cuh"

namespace momed {

namespace {

struct RecipeView {
    int32_t dim, Nc_mix;
    double G[3];
    double sys_size;
    const double* kcoord;    // [Nk][dim]
    const double* shift;     // [Ncc][dim]
    double p[8];
};

__device__ __forceinline__ void coord(const RecipeView& R, int k, int comp, double* out) {
    const int cc = (comp - 1) / R.Nc_mix;
    for (int d = 0; d < R.dim; ++d) {
        const double kv = R.kcoord[k * R.dim + d], sv = R.shift[cc * R.dim + d];
        out[d] = R.G[d] != 0.0 ? kv / R.G[d] + sv / R.G[d] : kv + sv;
    }
}

__device__ __forceinline__ double vff(const RecipeView& R, double q1, double q2) {
    const double Gl = R.p[0], D = R.p[1], W0 = R.p[2], ang = R.p[3];
    const double ql = sqrt(q1 * q1 + q2 * q2 + 2.0 * cos(ang) * q1 * q2) * Gl;
    if (ql == 0.0) return W0 * D;
    return W0 / ql * tanh(ql * D) * exp(-0.5 * (ql * ql));
}

__device__ __forceinline__ int ita(int g1, int g2) { return ((g1 & 1) == 0 && (g2 & 1) == 0) ? 1 : -1; }

__device__ __forceinline__ double cross(double a1, double a2, double b1, double b2) { return a1 * b2 - a2 * b1; }

// H_two(kf1, kf2, ki2, ki1) of the Landau-level recipe (2D coordinates)
__device__ double2 landau_v(const RecipeView& R, const double* kf1, const double* kf2, const double* ki2,
                            const double* ki1) {
    const int ns = (int)R.p[4];
    double q[2];
    int gs1[2], gs2[2];
    for (int i = 0; i < 2; ++i) {
        const double d = ki1[i] - kf1[i];
        q[i] = d - rint(d);                                   // rem(d, 1, RoundNearest)
    }
    for (int i = 0; i < 2; ++i) {
        gs1[i] = (int)rint(ki1[i] - kf1[i] - q[i]);
        gs2[i] = (int)rint(kf2[i] - ki2[i] - q[i]);
    }
    double vr = 0.0, vi = 0.0;
    for (int g1 = -ns; g1 <= ns; ++g1)
        for (int g2 = -ns; g2 <= ns; ++g2) {
            if (abs(g1 - g2) > ns) continue;
            const double qq1 = q[0] + g1, qq2 = q[1] + g2;
            double pa = 0.5 * cross(ki1[0], ki1[1], kf1[0], kf1[1]);
            pa += 0.5 * cross(ki1[0] + kf1[0], ki1[1] + kf1[1], qq1, qq2);
            pa += 0.5 * cross(ki2[0], ki2[1], kf2[0], kf2[1]);
            pa += 0.5 * cross(ki2[0] + kf2[0], ki2[1] + kf2[1], -qq1, -qq2);
            double s, c;
            sincospi(2.0 * pa, &s, &c);
            const int sg = ita(g1 + gs1[0], g2 + gs1[1]) * ita(g1 + gs2[0], g2 + gs2[1]);
            const double v = vff(R, qq1, qq2);
            vr += (sg * c) * v;
            vi += (sg * s) * v;
        }
    return make_double2(vr, vi);
}

// one upper term per thread: its raw contributions (direct - exchange) / sys_size, signed,
// conjugated or reduced to the real part as the normal ordering did, summed in merge order
__global__ void k_recipe_upper(RecipeView R, const int32_t* __restrict__ raw, const int64_t* __restrict__ start,
                               int64_t nupper, double2* __restrict__ out) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < nupper; u += (int64_t)gridDim.x * blockDim.x) {
        double ar = 0.0, ai = 0.0;
        for (int64_t c = start[u]; c < start[u + 1]; ++c) {
            const int32_t* r = raw + c * 9;
            double cf1[3], cf2[3], ci2[3], ci1[3];
            coord(R, r[0], r[4], cf1);
            coord(R, r[1], r[5], cf2);
            coord(R, r[2], r[6], ci2);
            coord(R, r[3], r[7], ci1);
            const double2 d = landau_v(R, cf1, cf2, ci2, ci1);
            const double2 e = landau_v(R, cf1, cf2, ci1, ci2);
            double xr = (d.x - e.x) / R.sys_size, xi = (d.y - e.y) / R.sys_size;
            const int fl = r[8];
            if (fl & 1) { xr = -xr; xi = -xi; }
            const int mode = (fl >> 1) & 3;
            if (mode == 1) xi = -xi;
            else if (mode == 2) xi = 0.0;
            ar += xr;
            ai += xi;
        }
        out[u] = make_double2(ar, ai);
    }
}

__global__ void k_recipe_slots(const double2* __restrict__ up, const int32_t* __restrict__ slot_upper,
                               const int32_t* __restrict__ slot_partner, int64_t nslots, double2* __restrict__ amp,
                               float2* __restrict__ amp32) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nslots; q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = slot_upper[q];
        if (u < 0) continue;
        double2 v = up[u];
        if (slot_partner[q]) v.y = -v.y;
        amp[q] = v;
        amp32[q] = make_float2((float)v.x, (float)v.y);
    }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

}  // namespace

void set_twobody_recipe(momed_handle* h, const momed_para* p, int32_t kind, const double* params, int32_t nparams,
                        const int32_t* raw, int64_t nraw, const int64_t* upper_start, int64_t nupper,
                        const int64_t* entry_upper, const int32_t* entry_partner, int64_t nentries) {
    MOMED_REQUIRE(h->op_set, MOMED_ESTATE, "set the operator (momed_set_scatter) before its recipe");
    MOMED_REQUIRE(!h->op.has_b, MOMED_EINVAL, "a recipe describes a single operator, not H(u) = A + u B");
    MOMED_REQUIRE(kind == MOMED_RECIPE_LANDAU_COULOMB, MOMED_EINVAL, "unknown recipe");
    MOMED_REQUIRE(p && p->k_list && p->Gk && p->dim == 2, MOMED_EINVAL, "the Landau-level recipe needs a 2D mesh");
    MOMED_REQUIRE(params && nparams == 5 && params[4] >= 0 && params[4] <= 16, MOMED_EINVAL,
                  "params: [Gl, D, W0, angle, nshell (0..16)]");
    MOMED_REQUIRE(p->Nc_mix >= 1 && p->Nc_conserve >= 1 && p->Nk >= 1, MOMED_EINVAL, "bad EDPara");
    MOMED_REQUIRE(nentries == h->op.nterms && (int64_t)h->op_order.size() == nentries, MOMED_EINVAL,
                  "the recipe must describe every term of the working operator");
    MOMED_REQUIRE(nraw >= 0 && nupper >= 0 && raw && upper_start && entry_upper && entry_partner, MOMED_EINVAL,
                  "null recipe table");
    MOMED_REQUIRE(upper_start[0] == 0 && upper_start[nupper] == nraw, MOMED_EINVAL, "upper_start must span raw");
    for (int64_t u = 0; u < nupper; ++u)
        MOMED_REQUIRE(upper_start[u] <= upper_start[u + 1], MOMED_EINVAL, "upper_start must be monotone");
    const int Nc = p->Nc_mix * p->Nc_conserve;
    for (int64_t c = 0; c < nraw; ++c) {
        const int32_t* r = raw + c * 9;
        for (int j = 0; j < 4; ++j) MOMED_REQUIRE(r[j] >= 0 && r[j] < p->Nk, MOMED_EINVAL, "raw momentum index");
        for (int j = 4; j < 8; ++j) MOMED_REQUIRE(r[j] >= 1 && r[j] <= Nc, MOMED_EINVAL, "raw component index");
        MOMED_REQUIRE(((r[8] >> 1) & 3) <= 2, MOMED_EINVAL, "raw flags");
    }
    std::vector<int32_t> su(nentries), sp(nentries);
    for (int64_t q = 0; q < nentries; ++q) {
        const int64_t e = h->op_order[q];
        MOMED_REQUIRE(entry_upper[e] >= -1 && entry_upper[e] < nupper, MOMED_EINVAL, "entry_upper out of range");
        su[q] = (int32_t)entry_upper[e];
        sp[q] = entry_partner[e] ? 1 : 0;
    }
    TwoBodyRecipe& R = h->recipe;
    cudaStream_t st = h->stream;
    R.set = false;
    R.kind = kind;
    R.dim = p->dim;
    R.Nk = p->Nk;
    R.Nc_mix = p->Nc_mix;
    R.Ncc = p->Nc_conserve;
    bool all = true;
    for (int d = 0; d < p->dim; ++d) {
        R.Gk[d] = (double)p->Gk[d];
        all = all && p->Gk[d] != 0;
    }
    R.sys_size = all ? (double)p->Nk : 1.0;             // scat_list.jl:437
    for (int i = 0; i < 8; ++i) R.params[i] = i < nparams ? params[i] : 0.0;
    R.nraw = nraw;
    R.nupper = nupper;
    std::vector<double> kc((size_t)p->Nk * p->dim);
    for (int i = 0; i < p->Nk; ++i)
        for (int d = 0; d < p->dim; ++d) kc[(size_t)i * p->dim + d] = (double)p->k_list[d + p->dim * i];
    auto up = [&](auto& dst, const auto* src, size_t count) {
        using T = std::decay_t<decltype(*src)>;
        dst.resize(std::max<size_t>(count, 1));
        if (count) MOMED_CUDA_TRY(cudaMemcpyAsync(dst.p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    };
    up(R.kcoord, kc.data(), kc.size());
    up(R.raw, raw, (size_t)nraw * 9);
    up(R.upper_start, upper_start, (size_t)nupper + 1);
    up(R.slot_upper, su.data(), su.size());
    up(R.slot_partner, sp.data(), sp.size());
    R.upper_amp.resize(std::max<int64_t>(nupper, 1));
    R.shift.resize((size_t)R.Ncc * R.dim);
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    R.set = true;
}

void set_kshift(momed_handle* h, const double* kshift) {
    TwoBodyRecipe& R = h->recipe;
    MOMED_REQUIRE(R.set && h->op_set, MOMED_ESTATE, "no recipe on the working operator (momed_set_twobody_recipe)");
    cudaStream_t st = h->stream;
    std::vector<double> sh((size_t)R.Ncc * R.dim, 0.0);
    if (kshift)
        for (size_t i = 0; i < sh.size(); ++i) {
            MOMED_REQUIRE(std::isfinite(kshift[i]), MOMED_EINVAL, "kshift must be finite");
            sh[i] = kshift[i];
        }
    MOMED_CUDA_TRY(cudaMemcpyAsync(R.shift.p, sh.data(), sh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    RecipeView V{};
    V.dim = R.dim;
    V.Nc_mix = R.Nc_mix;
    for (int d = 0; d < 3; ++d) V.G[d] = R.Gk[d];
    V.sys_size = R.sys_size;
    V.kcoord = R.kcoord.p;
    V.shift = R.shift.p;
    for (int i = 0; i < 8; ++i) V.p[i] = R.params[i];
    if (R.nupper > 0) {
        k_recipe_upper<<<grid_for(R.nupper), 256, 0, st>>>(V, R.raw.p, R.upper_start.p, R.nupper, R.upper_amp.p);
        k_recipe_slots<<<grid_for(h->op.nterms), 256, 0, st>>>(R.upper_amp.p, R.slot_upper.p, R.slot_partner.p,
                                                               h->op.nterms, h->op.amp.p, h->op.amp32.p);
        MOMED_CUDA_TRY(cudaGetLastError());
        note_launches(2);
    }
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));   // sh is read by the async copy
    h->sparse.release();                          // its values were built from the old amplitudes
    if (h->op.has_b) h->hcache.release();         // its runs are sorted by which parts are non-zero
}

}  // namespace momed
