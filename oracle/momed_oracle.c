/*
 * momed_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C, FP64 (and FP32 where the reference allows Float32) restatement of
 * MomentumED.jl's matrix-free Hamiltonian path.  It exists to check the CUDA
 * library: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm load it.  No product code links, imports or calls this file.
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the MomentumED.jl project root).  Parity pins: the EDCore unit-test known
 * answers (the EDCore/test files) are asserted against these functions in
 * tests/test_oracle_golden.py.  The eigensolver sits behind a third-party
 * boundary (KrylovKit.jl, compat 0.10.0 in MomentumED/Project.toml:27, not
 * vendored): it is restated here as a thick-restart (Krylov-Schur) Lanczos
 * and cross-checked against LAPACK (numpy.linalg.eigh) on dense matrices.
 *
 * Built with -ffp-contract=off so no multiply-add is fused: amplitudes are
 * then bit-identical to the same arithmetic done by Python floats and libm.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Scatter record shared with the Python wrapper (ctypes Structure).         */
/* ------------------------------------------------------------------------ */
typedef struct {
    double re, im;      /* Amp (Complex{F}; for F = Float32 it holds a float) */
    uint64_t out, in;   /* creation / annihilation masks (bit i-1 = orbital i) */
    uint64_t pm;        /* parity_mask(out) xor parity_mask(in) */
} or_scat;

typedef struct {
    int32_t dim, Nk, Nc_mix, Nc_conserve;
    const int64_t* k_list;   /* k_list[d + dim*i], i = 0..Nk-1 (Julia k_list[:, i+1]) */
    const int64_t* Gk;       /* [dim]; 0 means no periodicity */
} or_para;

/* Julia shift semantics: UInt64(1) << s is 0 for s >= 64. */
static inline uint64_t jl_one_shl(int s) { return (s >= 64 || s < 0) ? 0ULL : (1ULL << s); }
static inline int jl_tz(uint64_t x) { return x ? __builtin_ctzll(x) : 64; }

/* EDCore/src/types/scattering.jl:7-18 */
OR_API uint64_t or_parity_mask(uint64_t occ) {
    uint64_t mask = 0;
    while (occ > 0) {
        int tz1 = jl_tz(occ);
        occ &= occ - 1ULL;
        int tz2 = jl_tz(occ);
        occ &= occ - 1ULL;               /* occ == 0 stays 0 (wrapping 0 & ~0) */
        mask += jl_one_shl(tz2);
        mask -= jl_one_shl(tz1 + 1);
    }
    return mask;
}

/* EDCore/src/types/manybodystate_basis.jl:397-408 (mask form) */
OR_API int or_scat_occ_number(uint64_t n, uint64_t imask) {
    return __builtin_popcountll(n & or_parity_mask(imask));
}
/* manybodystate_basis.jl:439-449 (single orbital i, 1-based) */
OR_API int or_scat_occ_number_1(uint64_t n, int i, int bits) {
    if (i == bits) return 0;
    uint64_t mask = ~0ULL - jl_one_shl(i) + 1ULL;
    return __builtin_popcountll(n & mask);
}
/* manybodystate_basis.jl:450-458 (pair, 1-based) */
OR_API int or_scat_occ_number_2(uint64_t n, int i, int j) {
    int imin = i < j ? i : j, imax = i < j ? j : i;
    uint64_t mask = jl_one_shl(imax - 1) - jl_one_shl(imin);
    return __builtin_popcountll(n & mask);
}

/* ------------------------------------------------------------------------ */
/* Complex helpers with Julia's operation order (no fused multiply-add).    */
/* ------------------------------------------------------------------------ */
static inline void cmul(double ar, double ai, double br, double bi, double* r, double* i) {
    *r = ar * br - ai * bi;
    *i = ar * bi + ai * br;
}
static inline void cmulf(float ar, float ai, float br, float bi, float* r, float* i) {
    *r = ar * br - ai * bi;
    *i = ar * bi + ai * br;
}

/* ------------------------------------------------------------------------ */
/* Scatter constructors: EDCore/src/types/scattering.jl:52-153              */
/* ------------------------------------------------------------------------ */
static void scat_finish(or_scat* s, double re, double im, uint64_t out, uint64_t in) {
    s->re = re; s->im = im; s->out = out; s->in = in;
    s->pm = or_parity_mask(out) ^ or_parity_mask(in);   /* scattering.jl:60 */
}

/* One-body Scatter(V, i, j; upper_hermitian): scattering.jl:101-120 */
OR_API void or_scatter_1(double re, double im, int i, int j, int upper, or_scat* s) {
    uint64_t i_mask = jl_one_shl(i - 1), j_mask = jl_one_shl(j - 1);
    if (upper) {
        if (j_mask < i_mask) { uint64_t t = i_mask; i_mask = j_mask; j_mask = t; im = -im; }
        else if (j_mask == i_mask) { im = 0.0; }
    }
    scat_finish(s, re, im, i_mask, j_mask);
}

/* Two-body Scatter(V, i1, i2, j2, j1; upper_hermitian): scattering.jl:121-153 */
OR_API void or_scatter_2(double re, double im, int i1, int i2, int j2, int j1, int upper, or_scat* s) {
    uint64_t i_mask = jl_one_shl(i1 - 1) | jl_one_shl(i2 - 1);
    uint64_t j_mask = jl_one_shl(j1 - 1) | jl_one_shl(j2 - 1);
    if (j1 == j2 || i1 == i2) { scat_finish(s, 0.0, 0.0, i_mask, j_mask); return; }
    if (i1 < i2) { re = -re; im = -im; }
    if (j1 < j2) { re = -re; im = -im; }
    if (upper) {
        if (j_mask < i_mask) { uint64_t t = i_mask; i_mask = j_mask; j_mask = t; im = -im; }
        else if (j_mask == i_mask) { im = 0.0; }
    }
    scat_finish(s, re, im, i_mask, j_mask);
}

/* parity of the permutation that sorts v descending = parity of #pairs a<b with v[a]<v[b] */
static int desc_sort_parity(const int64_t* v, int n) {
    int inv = 0;
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b)
            if (v[a] < v[b]) inv ^= 1;
    return inv;
}

/* Generic N-body Scatter(V, out_in...; upper_hermitian): scattering.jl:63-100 */
OR_API int or_scatter_n(double re, double im, const int64_t* out_in, int n2, int upper, or_scat* s) {
    if (n2 % 2 != 0 || n2 > 128) return -1;
    int N = n2 / 2;
    int64_t is[64], js[64];
    for (int a = 0; a < N; ++a) is[a] = out_in[a];
    for (int a = 0; a < N; ++a) js[a] = out_in[n2 - 1 - a];          /* out_in[2N:-1:N+1] */
    uint64_t i_mask = 0, j_mask = 0;
    for (int a = 0; a < N; ++a) { i_mask |= jl_one_shl((int)is[a] - 1); j_mask |= jl_one_shl((int)js[a] - 1); }
    if (__builtin_popcountll(i_mask) < N || __builtin_popcountll(j_mask) < N) {
        scat_finish(s, 0.0, 0.0, i_mask, j_mask);
        return 0;
    }
    if ((desc_sort_parity(is, N) + desc_sort_parity(js, N)) & 1) { re = -re; im = -im; }
    if (upper) {
        if (j_mask < i_mask) { uint64_t t = i_mask; i_mask = j_mask; j_mask = t; im = -im; }
        else if (j_mask == i_mask) { im = 0.0; }
    }
    scat_finish(s, re, im, i_mask, j_mask);
    return 0;
}

/* scattering.jl:170 */
OR_API int or_isupper(const or_scat* s) {
    return s->in > s->out || (s->in == s->out && s->im == 0.0);
}

/* Stable sort by (in, out): scattering.jl:205-207 (isless) with Julia's stable default sort */
static int scat_less(const or_scat* a, const or_scat* b) {
    return a->in < b->in || (a->in == b->in && a->out < b->out);
}
static void merge_sort_scat(or_scat* a, or_scat* tmp, int64_t n) {
    if (n < 2) return;
    int64_t h = n / 2;
    merge_sort_scat(a, tmp, h);
    merge_sort_scat(a + h, tmp, n - h);
    int64_t i = 0, j = h, k = 0;
    while (i < h && j < n) {
        if (scat_less(&a[j], &a[i])) tmp[k++] = a[j++];   /* take right only if strictly less: stable */
        else tmp[k++] = a[i++];
    }
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, (size_t)n * sizeof(or_scat));
}
OR_API void or_sort_scat(or_scat* list, int64_t n) {
    if (n < 2) return;
    or_scat* tmp = (or_scat*)malloc((size_t)n * sizeof(or_scat));
    merge_sort_scat(list, tmp, n);
    free(tmp);
}

/* sort_merge_scatlist: scattering.jl:258-277.  prec = 64 or 32 (Complex{Float32} arithmetic).
 * Returns the merged length, or -1 if check_upper fails. out may alias nothing; capacity n. */
OR_API int64_t or_sort_merge(const or_scat* list, int64_t n, int check_upper, int prec, or_scat* out) {
    if (n == 0) return 0;
    if (check_upper)
        for (int64_t i = 0; i < n; ++i)
            if (!or_isupper(&list[i])) return -1;
    or_scat* sorted = (or_scat*)malloc((size_t)n * sizeof(or_scat));
    memcpy(sorted, list, (size_t)n * sizeof(or_scat));
    or_sort_scat(sorted, n);
    /* merged_list = [0.0 * sorted_list[1]] */
    int64_t m = 0;
    out[0] = sorted[0];
    if (prec == 32) {
        float r, i;
        cmulf(0.0f, 0.0f, (float)sorted[0].re, (float)sorted[0].im, &r, &i);
        out[0].re = r; out[0].im = i;
    } else {
        double r, i;
        cmul(0.0, 0.0, sorted[0].re, sorted[0].im, &r, &i);
        out[0].re = r; out[0].im = i;
    }
    m = 1;
    for (int64_t k = 0; k < n; ++k) {
        or_scat* last = &out[m - 1];
        if (sorted[k].in == last->in && sorted[k].out == last->out) {
            if (prec == 32) {
                last->re = (double)((float)last->re + (float)sorted[k].re);
                last->im = (double)((float)last->im + (float)sorted[k].im);
            } else {
                last->re = last->re + sorted[k].re;
                last->im = last->im + sorted[k].im;
            }
        } else {
            out[m++] = sorted[k];
        }
    }
    free(sorted);
    return m;
}

/* LinearMap construction for an upper_hermitian operator: linear_map.jl:22-32.
 * out capacity >= 2n.  Appends s' (scattering.jl:185-187) for every non-diagonal term, stable sort. */
OR_API int64_t or_hermitian_complete(const or_scat* upper, int64_t n, or_scat* out) {
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) out[m++] = upper[i];
    for (int64_t i = 0; i < n; ++i) {
        if (upper[i].in != upper[i].out) {
            or_scat a;
            a.re = upper[i].re; a.im = -upper[i].im;
            a.out = upper[i].in; a.in = upper[i].out;
            a.pm = or_parity_mask(a.out) ^ or_parity_mask(a.in);
            out[m++] = a;
        }
    }
    or_sort_scat(out, m);
    return m;
}

/* ------------------------------------------------------------------------ */
/* Colex enumeration: EDCore/src/colex_mbslist.jl                           */
/* ------------------------------------------------------------------------ */
OR_API int64_t or_binomial(int64_t n, int64_t k) {
    if (k < 0 || n < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    int64_t r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

/* colex_mbslist.jl:2-21; writes t sorted 1-based positions, returns count (0 on the early returns) */
OR_API int or_unrank_colex(int n, int t, int64_t k, int64_t* out) {
    if (t == 0 || k <= 0 || k > or_binomial(n, t)) return 0;
    int64_t x = k - 1;
    int len = 0;
    for (int i = t; i >= 1; --i) {
        int64_t c = i - 1;
        while (c + 1 < n && or_binomial(c + 1, i) <= x) c += 1;
        out[len++] = c + 1;
        x -= or_binomial(c, i);
    }
    /* sort! ascending */
    for (int a = 1; a < len; ++a) {
        int64_t v = out[a]; int b = a - 1;
        while (b >= 0 && out[b] > v) { out[b + 1] = out[b]; --b; }
        out[b + 1] = v;
    }
    return len;
}

/* ColexMBS64 / ColexMBS64Mask iteration (colex_mbslist.jl:39-91, 111-173).
 * start >= 1, end inclusive (1-based numbers, as the Julia constructors).
 * mask == NULL means the plain ColexMBS64(n, t, start, end).  Returns count; writes
 * up to cap states into out (out may be NULL to count). */
static int64_t colex_run(int n, int t, const int64_t* mask, int mlen, int64_t start, int64_t end,
                         uint64_t* out, int64_t cap) {
    int len = mask ? mlen : n;
    int64_t full = or_binomial(len, t);
    if (start < 1) return -1;
    if (start > full || end < start) return 0;
    if (end > full) end = full;
    int64_t s[66];
    if (start == 1) { for (int i = 0; i < t; ++i) s[i] = i + 1; }
    else { or_unrank_colex(len, t, start, s); }
    s[t] = len + 1;
    int64_t count = 0;
    for (int64_t num = start; num <= end; ++num) {
        if (num > start) {
            /* successor rule (colex_mbslist.jl:81-89) */
            int done = 0;
            for (int i = 0; i < t; ++i) {
                if (s[i] < s[i + 1] - 1) {
                    s[i] += 1;
                    for (int j = 0; j < i; ++j) s[j] = j + 1;
                    done = 1;
                    break;
                }
            }
            if (!done) break;
        }
        uint64_t st = 0;
        for (int i = 0; i < t; ++i) {
            int64_t orb = mask ? mask[s[i] - 1] : s[i];
            st |= jl_one_shl((int)orb - 1);
        }
        if (out && count < cap) out[count] = st;
        ++count;
    }
    return count;
}
OR_API int64_t or_colex(int n, int t, int64_t start, int64_t end, uint64_t* out, int64_t cap) {
    return colex_run(n, t, NULL, 0, start, end, out, cap);
}
OR_API int64_t or_colex_mask(int n, int t, const int64_t* mask, int mlen, int64_t start, int64_t end,
                             uint64_t* out, int64_t cap) {
    return colex_run(n, t, mask, mlen, start, end, out, cap);
}

/* ------------------------------------------------------------------------ */
/* Momentum sectors: MomentumED/src/preparation/momentum_decomposition.jl   */
/* ------------------------------------------------------------------------ */
static int64_t jl_mod(int64_t a, int64_t g) { int64_t r = a % g; return r < 0 ? r + g : r; }

/* init_parameter.jl:148-152 */
static void momentum_residue(int dim, const int64_t* k, const int64_t* Gk, int64_t* out) {
    for (int d = 0; d < dim; ++d) out[d] = Gk[d] == 0 ? k[d] : jl_mod(k[d], Gk[d]);
}

/* momentum_decomposition.jl:49-59 (MBS_totalmomentum on a state of one component) */
static void state_momentum(const or_para* p, uint64_t st, int64_t* out) {
    int64_t k[8] = {0};
    while (st) {
        int tz = __builtin_ctzll(st);
        st &= st - 1;
        int i = tz + 1;
        int ik = (i - 1) % p->Nk;             /* mod1(i, Nk) - 1 */
        for (int d = 0; d < p->dim; ++d) k[d] += p->k_list[d + p->dim * ik];
    }
    momentum_residue(p->dim, k, p->Gk, out);
}

typedef struct { uint64_t* v; int64_t n, cap; } u64vec;
static void u64push(u64vec* a, uint64_t x) {
    if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 64; a->v = (uint64_t*)realloc(a->v, (size_t)a->cap * 8); }
    a->v[a->n++] = x;
}

typedef struct {
    const or_para* p;
    const int64_t* mom_list;   /* [nmom*dim] */
    int nmom;
    u64vec* lists;             /* [nmom] */
} sub_ctx;

/* momentum_decomposition.jl:101-152 */
static void recurse(sub_ctx* c, const int64_t* N_each, int ncomp, uint64_t acc, const int64_t* acc_k,
                    const int64_t* mask, int mlen, int64_t start, int64_t end) {
    const or_para* p = c->p;
    int dim = p->dim;
    if (ncomp > 0) {
        int nbits = p->Nk * p->Nc_mix;
        int64_t Nlast = N_each[ncomp - 1];
        int t = (int)(Nlast < 0 ? -Nlast : Nlast);
        int sgn = Nlast > 0 ? 1 : (Nlast < 0 ? -1 : 0);
        const int64_t* mthis = NULL; int mthis_len = 0; int64_t mbuf[64];
        const int64_t* mrest = NULL; int mrest_len = 0;
        if (mask) {
            int64_t ncomp_orb = (int64_t)nbits * (ncomp - 1);
            int i = 0;   /* searchsortedlast */
            while (i < mlen && mask[i] <= ncomp_orb) ++i;
            mthis_len = mlen - i;
            for (int a = 0; a < mthis_len; ++a) mbuf[a] = mask[i + a] - ncomp_orb;
            mthis = mbuf; mrest = mask; mrest_len = i;
        }
        int len = mask ? mthis_len : nbits;
        int64_t full = or_binomial(len, t);
        if (start < 1) start = 1;
        if (end > full) end = full;
        if (start > end) return;
        uint64_t* states = (uint64_t*)malloc((size_t)(end - start + 1) * 8);
        int64_t ns = colex_run(nbits, t, mthis, mthis_len, start, end, states, end - start + 1);
        for (int64_t s = 0; s < ns; ++s) {
            int64_t km[8], nk[8];
            state_momentum(p, states[s], km);
            for (int d = 0; d < dim; ++d) nk[d] = acc_k[d] + sgn * km[d];
            uint64_t nacc = (nbits >= 64 ? 0 : (acc << nbits)) | states[s];
            recurse(c, N_each, ncomp - 1, nacc, nk, mask ? mrest : NULL, mrest_len, 1, INT64_MAX);
        }
        free(states);
    } else {
        int64_t k[8];
        momentum_residue(dim, acc_k, p->Gk, k);
        for (int s = 0; s < c->nmom; ++s) {
            int eq = 1;
            for (int d = 0; d < dim; ++d) if (c->mom_list[s * dim + d] != k[d]) { eq = 0; break; }
            if (eq) { u64push(&c->lists[s], acc); break; }
        }
    }
}

/* ED_momentum_subspaces: momentum_decomposition.jl:188-262.
 * mask (sorted) may be NULL; mom_restrict != 0 uses mom_in[nmom_in*dim].
 * Two-call protocol: pass out_basis == NULL to get *n_sectors and the total; then call again
 * with buffers out_sector_k[nsec*dim], out_sizes[nsec], out_basis[total]. */
OR_API int64_t or_momentum_subspaces(const or_para* p, const int64_t* N_each, int ncc,
                                     const int64_t* mask, int mlen,
                                     int mom_restrict, const int64_t* mom_in, int nmom_in,
                                     int64_t* out_sector_k, int64_t* out_sizes, uint64_t* out_basis,
                                     int64_t* n_sectors) {
    int dim = p->dim;
    if (ncc != p->Nc_conserve || dim < 1 || dim > 8) return -1;
    int64_t* mom = NULL; int nmom = 0;
    if (mom_restrict) {
        mom = (int64_t*)malloc((size_t)(nmom_in > 0 ? nmom_in : 1) * dim * 8);
        for (int s = 0; s < nmom_in; ++s) {
            int64_t r[8];
            momentum_residue(dim, &mom_in[s * dim], p->Gk, r);
            int dup = 0;
            for (int u = 0; u < nmom && !dup; ++u) {
                int eq = 1;
                for (int d = 0; d < dim; ++d) if (mom[u * dim + d] != r[d]) { eq = 0; break; }
                dup = eq;
            }
            if (!dup) { memcpy(&mom[nmom * dim], r, (size_t)dim * 8); ++nmom; }
        }
    } else {
        int64_t lo[8], cnt[8];
        int64_t Ntot = 0;
        for (int c = 0; c < ncc; ++c) Ntot += N_each[c];
        nmom = 1;
        for (int d = 0; d < dim; ++d) {
            if (p->Gk[d] == 0) {
                int64_t mn = INT64_MAX, mx = INT64_MIN;
                for (int i = 0; i < p->Nk; ++i) {
                    int64_t v = p->k_list[d + dim * i];
                    if (v < mn) mn = v;
                    if (v > mx) mx = v;
                }
                lo[d] = mn * Ntot;
                cnt[d] = mx * Ntot - mn * Ntot + 1;
                if (cnt[d] < 0) cnt[d] = 0;
            } else { lo[d] = 0; cnt[d] = p->Gk[d]; }
            nmom *= (int)cnt[d];
        }
        mom = (int64_t*)malloc((size_t)(nmom > 0 ? nmom : 1) * dim * 8);
        for (int s = 0; s < nmom; ++s) {          /* Iterators.product: first coordinate fastest */
            int r = s;
            for (int d = 0; d < dim; ++d) { mom[s * dim + d] = lo[d] + r % cnt[d]; r /= (int)cnt[d]; }
        }
    }
    int64_t* sorted_mask = NULL;
    if (mask && mlen >= 0) {
        sorted_mask = (int64_t*)malloc((size_t)(mlen > 0 ? mlen : 1) * 8);
        memcpy(sorted_mask, mask, (size_t)mlen * 8);
        for (int a = 1; a < mlen; ++a) {
            int64_t v = sorted_mask[a]; int b = a - 1;
            while (b >= 0 && sorted_mask[b] > v) { sorted_mask[b + 1] = sorted_mask[b]; --b; }
            sorted_mask[b + 1] = v;
        }
    }
    sub_ctx c;
    c.p = p; c.mom_list = mom; c.nmom = nmom;
    c.lists = (u64vec*)calloc((size_t)(nmom > 0 ? nmom : 1), sizeof(u64vec));
    int64_t zero[8] = {0};
    recurse(&c, N_each, ncc, 0ULL, zero, sorted_mask, sorted_mask ? mlen : 0, 1, INT64_MAX);
    /* HilbertSubspace sorts an unsorted list (hilbert_subspace.jl:24-27) */
    int64_t nsec = 0, total = 0;
    for (int s = 0; s < nmom; ++s) {
        u64vec* L = &c.lists[s];
        int sorted = 1;
        for (int64_t i = 1; i < L->n; ++i) if (L->v[i] < L->v[i - 1]) { sorted = 0; break; }
        if (!sorted) {
            for (int64_t a = 1; a < L->n; ++a) {
                uint64_t v = L->v[a]; int64_t b = a - 1;
                while (b >= 0 && L->v[b] > v) { L->v[b + 1] = L->v[b]; --b; }
                L->v[b + 1] = v;
            }
        }
        if (L->n > 0) {
            if (out_basis) {
                memcpy(&out_sector_k[nsec * dim], &mom[s * dim], (size_t)dim * 8);
                out_sizes[nsec] = L->n;
                memcpy(&out_basis[total], L->v, (size_t)L->n * 8);
            }
            ++nsec; total += L->n;
        }
        free(L->v);
    }
    free(c.lists); free(mom); free(sorted_mask);
    *n_sectors = nsec;
    return total;
}

/* ------------------------------------------------------------------------ */
/* Scatter-list builders: MomentumED/src/preparation/scat_list.jl           */
/* Index mode (H_one(k, cf, ci), H_two(kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1))     */
/* and float-coordinate mode (coordinates k/Gk as doubles plus per-component shift). */
/* ------------------------------------------------------------------------ */
typedef void (*or_h1_fn)(void* ctx, int64_t k, int64_t cf, int64_t ci, double* re, double* im);
typedef void (*or_h2_fn)(void* ctx, int64_t kf1, int64_t kf2, int64_t ki2, int64_t ki1,
                         int64_t cf1, int64_t cf2, int64_t ci2, int64_t ci1, double* re, double* im);
typedef void (*or_h1c_fn)(void* ctx, const double* k, int64_t cf, int64_t ci, double* re, double* im);
typedef void (*or_h2c_fn)(void* ctx, const double* kf1, const double* kf2, const double* ki2, const double* ki1,
                          int64_t cf1, int64_t cf2, int64_t ci2, int64_t ci1, double* re, double* im);
/* Rational-coordinate mode (scat_list.jl:5-16, the default when kshift is nothing, an integer
 * or a rational): each coordinate is passed as an exact fraction, k[2d] / k[2d + 1] for
 * direction d (not reduced), k/Gk + shift/Gk where Gk != 0 and k + shift where Gk == 0; the
 * shift of conserved component c is rshift[2(d + dim c)] / rshift[2(d + dim c) + 1]. */
typedef void (*or_h1r_fn)(void* ctx, const int64_t* k, int64_t cf, int64_t ci, double* re, double* im);
typedef void (*or_h2r_fn)(void* ctx, const int64_t* kf1, const int64_t* kf2, const int64_t* ki2, const int64_t* ki1,
                          int64_t cf1, int64_t cf2, int64_t ci2, int64_t ci1, double* re, double* im);

/* exact coordinate of momentum index k (1-based) of conserved component cc (1-based) */
static void rational_coord(const or_para* p, const int64_t* rshift, int k, int cc, int64_t* out) {
    for (int d = 0; d < p->dim; ++d) {
        int64_t kv = p->k_list[d + p->dim * (k - 1)];
        int64_t sn = rshift ? rshift[2 * (d + p->dim * (cc - 1))] : 0;
        int64_t sd = rshift ? rshift[2 * (d + p->dim * (cc - 1)) + 1] : 1;
        int64_t g = p->Gk[d] != 0 ? p->Gk[d] : 1;
        out[2 * d] = kv * sd + sn;
        out[2 * d + 1] = g * sd;
    }
}

static int64_t push_scat(or_scat* out, int64_t cap, int64_t n, const or_scat* s) {
    if (out && n < cap) out[n] = *s;
    return n + 1;
}

/* scat_list.jl:78-142 (index mode at 126-138, coordinate mode at 92-118).
 * prec 32 rounds H_one's value to Complex{Float32}.  Returns the sorted-merged count,
 * the merged list in out (capacity cap); when out == NULL it returns the raw term count. */
static int64_t onebody_common(const or_para* p, or_h1_fn f, or_h1c_fn fc, or_h1r_fn fr, void* ctx,
                              const double* shift /* [dim*Ncc] or NULL */, const int64_t* rshift, int prec,
                              or_scat* out, int64_t cap) {
    int Nk = p->Nk, Ncm = p->Nc_mix, Ncc = p->Nc_conserve, dim = p->dim;
    int64_t n = 0;
    int64_t rawcap = (int64_t)Ncc * Ncm * Ncm * Nk;
    or_scat* raw = (or_scat*)malloc((size_t)(rawcap > 0 ? rawcap : 1) * sizeof(or_scat));
    for (int cc = 1; cc <= Ncc; ++cc)
        for (int cmi = 1; cmi <= Ncm; ++cmi)
            for (int cmf = 1; cmf <= Ncm; ++cmf) {
                int cf = cmf + (cc - 1) * Ncm, ci = cmi + (cc - 1) * Ncm;
                for (int k = 1; k <= Nk; ++k) {
                    int i_out = k + Nk * (cf - 1), i_in = k + Nk * (ci - 1);
                    if (i_in >= i_out) {
                        double re = 0, im = 0;
                        if (fr) {
                            int64_t kr[16];
                            rational_coord(p, rshift, k, cc, kr);
                            fr(ctx, kr, cf, ci, &re, &im);
                        } else if (fc) {
                            double kc[8];
                            for (int d = 0; d < dim; ++d) {
                                double kv = (double)p->k_list[d + dim * (k - 1)];
                                double sv = shift ? shift[d + dim * (cc - 1)] : 0.0;
                                if (p->Gk[d] != 0) { kv = kv / (double)p->Gk[d]; sv = sv / (double)p->Gk[d]; }
                                kc[d] = kv + sv;
                            }
                            fc(ctx, kc, cf, ci, &re, &im);
                        } else {
                            f(ctx, k, cf, ci, &re, &im);
                        }
                        if (prec == 32) { re = (float)re; im = (float)im; }
                        if (!(re == 0.0 && im == 0.0)) {
                            or_scat s;
                            or_scatter_1(re, im, i_out, i_in, 1, &s);
                            n = push_scat(raw, rawcap, n, &s);
                        }
                    }
                }
            }
    if (!out) { free(raw); return n; }
    or_scat* merged = (or_scat*)malloc((size_t)(n > 0 ? n : 1) * sizeof(or_scat));
    int64_t m = or_sort_merge(raw, n, 1, prec, merged);
    if (m > cap) m = -2;
    else if (m > 0) memcpy(out, merged, (size_t)m * sizeof(or_scat));
    free(raw); free(merged);
    return m;
}
OR_API int64_t or_scatterlist_onebody(const or_para* p, or_h1_fn f, void* ctx, int prec, or_scat* out, int64_t cap) {
    return onebody_common(p, f, NULL, NULL, ctx, NULL, NULL, prec, out, cap);
}
OR_API int64_t or_scatterlist_onebody_coord(const or_para* p, or_h1c_fn f, void* ctx, const double* shift,
                                            int prec, or_scat* out, int64_t cap) {
    return onebody_common(p, NULL, f, NULL, ctx, shift, NULL, prec, out, cap);
}
OR_API int64_t or_scatterlist_onebody_rational(const or_para* p, or_h1r_fn f, void* ctx, const int64_t* rshift,
                                               int prec, or_scat* out, int64_t cap) {
    return onebody_common(p, NULL, NULL, f, ctx, NULL, rshift, prec, out, cap);
}

/* group_momentum_pairs: scat_list.jl:174-200.  Pairs (i, j), i >= j, 1-based, keyed by
 * the residue of k_i + k_j.  Group iteration order is irrelevant to the final sorted list
 * (each (in, out) key is produced once), so groups are walked in first-appearance order. */
typedef struct { int i, j; int64_t K[8]; } pair_t;

static int64_t twobody_common(const or_para* p, or_h2_fn f, or_h2c_fn fc, or_h2r_fn fr, void* ctx,
                              const double* shift, const int64_t* rshift, int prec, or_scat* out, int64_t cap) {
    int Nk = p->Nk, Nc = p->Nc_mix * p->Nc_conserve, Ncm = p->Nc_mix, dim = p->dim;
    int all_nonzero = 1;
    for (int d = 0; d < dim; ++d) if (p->Gk[d] == 0) all_nonzero = 0;
    int64_t sys_size = all_nonzero ? Nk : 1;                      /* scat_list.jl:437 */
    int npairs = Nk * (Nk + 1) / 2;
    pair_t* pairs = (pair_t*)malloc((size_t)npairs * sizeof(pair_t));
    int* group = (int*)malloc((size_t)npairs * sizeof(int));
    int ngroups = 0, np = 0;
    int64_t* gK = (int64_t*)malloc((size_t)npairs * dim * 8);
    for (int i = 1; i <= Nk; ++i)
        for (int j = 1; j <= i; ++j) {
            int64_t k[8];
            for (int d = 0; d < dim; ++d)
                k[d] = p->k_list[d + dim * (i - 1)] + p->k_list[d + dim * (j - 1)];
            pair_t* pr = &pairs[np];
            pr->i = i; pr->j = j;
            momentum_residue(dim, k, p->Gk, pr->K);
            int g = -1;
            for (int u = 0; u < ngroups && g < 0; ++u) {
                int eq = 1;
                for (int d = 0; d < dim; ++d) if (gK[u * dim + d] != pr->K[d]) { eq = 0; break; }
                if (eq) g = u;
            }
            if (g < 0) { g = ngroups++; memcpy(&gK[g * dim], pr->K, (size_t)dim * 8); }
            group[np++] = g;
        }
    int64_t rawcap = 1 << 16, n = 0;
    or_scat* raw = (or_scat*)malloc((size_t)rawcap * sizeof(or_scat));
    double kc[4][8];
    for (int g = 0; g < ngroups; ++g) {
        for (int a = 0; a < np; ++a) {
            if (group[a] != g) continue;
            int ki1 = pairs[a].i, ki2 = pairs[a].j;
            for (int b = 0; b < np; ++b) {
                if (group[b] != g) continue;
                int kf1 = pairs[b].i, kf2 = pairs[b].j;
                for (int ci1 = 1; ci1 <= Nc; ++ci1)
                for (int ci2 = 1; ci2 <= Nc; ++ci2)
                for (int cf1 = 1; cf1 <= Nc; ++cf1)
                for (int cf2 = 1; cf2 <= Nc; ++cf2) {
                    int f1 = kf1 + Nk * (cf1 - 1), f2 = kf2 + Nk * (cf2 - 1);
                    int i1 = ki1 + Nk * (ci1 - 1), i2 = ki2 + Nk * (ci2 - 1);
                    if (i1 == i2 || f1 == f2) continue;
                    if (ki1 == ki2 && i1 < i2) continue;
                    if (kf1 == kf2 && f1 < f2) continue;
                    int imin = i1 < i2 ? i1 : i2, imax = i1 < i2 ? i2 : i1;
                    int fmin = f1 < f2 ? f1 : f2, fmax = f1 < f2 ? f2 : f1;
                    if (!(imin > fmin || (imin == fmin && imax >= fmax))) continue;   /* minmax >= */
                    double dr, di, er, ei;
                    if (fr) {
                        int ks[4] = {kf1, kf2, ki2, ki1};
                        int cs[4] = {(cf1 - 1) / Ncm + 1, (cf2 - 1) / Ncm + 1, (ci2 - 1) / Ncm + 1, (ci1 - 1) / Ncm + 1};
                        int64_t kr[4][16];
                        for (int q = 0; q < 4; ++q) rational_coord(p, rshift, ks[q], cs[q], kr[q]);
                        fr(ctx, kr[0], kr[1], kr[2], kr[3], cf1, cf2, ci2, ci1, &dr, &di);
                        fr(ctx, kr[0], kr[1], kr[3], kr[2], cf1, cf2, ci1, ci2, &er, &ei);
                    } else if (fc) {
                        int ks[4] = {kf1, kf2, ki2, ki1};
                        int cs[4] = {(cf1 - 1) / Ncm + 1, (cf2 - 1) / Ncm + 1, (ci2 - 1) / Ncm + 1, (ci1 - 1) / Ncm + 1};
                        for (int q = 0; q < 4; ++q)
                            for (int d = 0; d < dim; ++d) {
                                double kv = (double)p->k_list[d + dim * (ks[q] - 1)];
                                double sv = shift ? shift[d + dim * (cs[q] - 1)] : 0.0;
                                if (p->Gk[d] != 0) { kv = kv / (double)p->Gk[d]; sv = sv / (double)p->Gk[d]; }
                                kc[q][d] = kv + sv;
                            }
                        fc(ctx, kc[0], kc[1], kc[2], kc[3], cf1, cf2, ci2, ci1, &dr, &di);
                        fc(ctx, kc[0], kc[1], kc[3], kc[2], cf1, cf2, ci1, ci2, &er, &ei);
                    } else {
                        f(ctx, kf1, kf2, ki2, ki1, cf1, cf2, ci2, ci1, &dr, &di);
                        f(ctx, kf1, kf2, ki1, ki2, cf1, cf2, ci1, ci2, &er, &ei);
                    }
                    double ar, ai;
                    if (prec == 32) {
                        float r = (float)dr - (float)er, im = (float)di - (float)ei;
                        r = r / (float)sys_size; im = im / (float)sys_size;
                        ar = r; ai = im;
                    } else {
                        ar = (dr - er) / (double)sys_size;
                        ai = (di - ei) / (double)sys_size;
                    }
                    if (!(ar == 0.0 && ai == 0.0)) {
                        or_scat s;
                        or_scatter_2(ar, ai, f1, f2, i2, i1, 1, &s);
                        if (n == rawcap) { rawcap *= 2; raw = (or_scat*)realloc(raw, (size_t)rawcap * sizeof(or_scat)); }
                        raw[n++] = s;
                    }
                }
            }
        }
    }
    free(pairs); free(group); free(gK);
    if (!out) { free(raw); return n; }
    or_scat* merged = (or_scat*)malloc((size_t)(n > 0 ? n : 1) * sizeof(or_scat));
    int64_t m = or_sort_merge(raw, n, 1, prec, merged);
    if (m > cap) m = -2;
    else if (m > 0) memcpy(out, merged, (size_t)m * sizeof(or_scat));
    free(raw); free(merged);
    return m;
}
OR_API int64_t or_scatterlist_twobody(const or_para* p, or_h2_fn f, void* ctx, int prec, or_scat* out, int64_t cap) {
    return twobody_common(p, f, NULL, NULL, ctx, NULL, NULL, prec, out, cap);
}
OR_API int64_t or_scatterlist_twobody_coord(const or_para* p, or_h2c_fn f, void* ctx, const double* shift,
                                            int prec, or_scat* out, int64_t cap) {
    return twobody_common(p, NULL, f, NULL, ctx, shift, NULL, prec, out, cap);
}
OR_API int64_t or_scatterlist_twobody_rational(const or_para* p, or_h2r_fn f, void* ctx, const int64_t* rshift,
                                               int prec, or_scat* out, int64_t cap) {
    return twobody_common(p, NULL, NULL, f, ctx, NULL, rshift, prec, out, cap);
}

/* ------------------------------------------------------------------------ */
/* Synthetic Hamiltonian recipe for the workload meshes (index mode).       */
/*   k-mesh a x b, k_list[:, i] = ((i-1) mod a, (i-1) div a), Gk = (a, b).   */
/*   H_one(k, cf, ci) = d(cf,ci) (cos(2 pi kx/a) + cos(2 pi ky/b))           */
/*   H_two(a1,a2,a3,a4,c...) = comp * exp(-|q|^2/2)/(|q|+0.5) * e^{i th}     */
/*     q = k(a3) - k(a1) folded per direction to the nearest image           */
/*     th tabulated once per {(a1a2a3a4),(a3a4a1a2)} in lexicographic order   */
/*     from SplitMix64(seed), th(a3a4a1a2) = -th(a1a2a3a4), self pairs th=0. */
/*     comp = d(cf1,ci1) d(cf2,ci2) + beta [cf1 != cf2] d(cf1,ci2) d(cf2,ci1) */
/*     beta = first draw of the stream.                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
    int32_t a, b, Nk, pad;
    double beta;
    double* theta;     /* Nk^4 */
} or_synth;

static uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double u01(uint64_t* s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

OR_API int or_synth_init(or_synth* S, int a, int b, uint64_t seed) {
    int Nk = a * b;
    S->a = a; S->b = b; S->Nk = Nk; S->pad = 0;
    size_t n4 = (size_t)Nk * Nk * Nk * Nk;
    S->theta = (double*)calloc(n4, sizeof(double));
    if (!S->theta) return -1;
    uint64_t st = seed;
    S->beta = u01(&st);
    for (int a1 = 0; a1 < Nk; ++a1)
    for (int a2 = 0; a2 < Nk; ++a2)
    for (int a3 = 0; a3 < Nk; ++a3)
    for (int a4 = 0; a4 < Nk; ++a4) {
        int x1 = a1 % a, y1 = a1 / a, x2 = a2 % a, y2 = a2 / a;
        int x3 = a3 % a, y3 = a3 / a, x4 = a4 % a, y4 = a4 / a;
        if (jl_mod(x1 + x2 - x3 - x4, a) != 0 || jl_mod(y1 + y2 - y3 - y4, b) != 0) continue;
        int lt = (a1 < a3) || (a1 == a3 && a2 < a4);
        int eq = (a1 == a3 && a2 == a4);
        size_t idx = (((size_t)a1 * Nk + a2) * Nk + a3) * Nk + a4;
        size_t pidx = (((size_t)a3 * Nk + a4) * Nk + a1) * Nk + a2;
        if (lt) {
            double th = 2.0 * M_PI * u01(&st);
            S->theta[idx] = th;
            S->theta[pidx] = -th;
        } else if (eq) {
            S->theta[idx] = 0.0;
        }
    }
    return 0;
}
OR_API void or_synth_free(or_synth* S) { free(S->theta); S->theta = NULL; }
OR_API double or_synth_beta(const or_synth* S) { return S->beta; }

static double fold_half(double t) { return t - floor(t + 0.5); }

OR_API void or_synth_h1(void* ctx, int64_t k, int64_t cf, int64_t ci, double* re, double* im) {
    or_synth* S = (or_synth*)ctx;
    if (cf != ci) { *re = 0.0; *im = 0.0; return; }
    int kx = (int)((k - 1) % S->a), ky = (int)((k - 1) / S->a);
    *re = cos(2.0 * M_PI * kx / S->a) + cos(2.0 * M_PI * ky / S->b);
    *im = 0.0;
}

OR_API void or_synth_h2(void* ctx, int64_t a1, int64_t a2, int64_t a3, int64_t a4,
                        int64_t cf1, int64_t cf2, int64_t ci2, int64_t ci1, double* re, double* im) {
    or_synth* S = (or_synth*)ctx;
    double comp = 0.0;
    if (cf1 == ci1 && cf2 == ci2) comp = comp + 1.0;
    if (cf1 != cf2 && cf1 == ci2 && cf2 == ci1) comp = comp + S->beta;
    if (comp == 0.0) { *re = 0.0; *im = 0.0; return; }
    int Nk = S->Nk;
    int qx = (int)((a3 - 1) % S->a) - (int)((a1 - 1) % S->a);
    int qy = (int)((a3 - 1) / S->a) - (int)((a1 - 1) / S->a);
    double fx = fold_half((double)qx / (double)S->a);
    double fy = fold_half((double)qy / (double)S->b);
    double qn = 2.0 * M_PI * sqrt(fx * fx + fy * fy);
    double mag = exp(-(qn * qn) / 2.0) / (qn + 0.5);
    double th = S->theta[(((size_t)(a1 - 1) * Nk + (a2 - 1)) * Nk + (a3 - 1)) * Nk + (a4 - 1)];
    double m = comp * mag;
    *re = m * cos(th);
    *im = m * sin(th);
}

/* Convenience: k_list of an a x b mesh (column i = ((i-1) mod a, (i-1) div a)). */
OR_API void or_mesh_klist(int a, int b, int64_t* k_list) {
    for (int i = 0; i < a * b; ++i) { k_list[2 * i] = i % a; k_list[2 * i + 1] = i / a; }
}
OR_API int64_t or_synth_onebody(const or_para* p, or_synth* S, int prec, or_scat* out, int64_t cap) {
    return onebody_common(p, or_synth_h1, NULL, NULL, S, NULL, NULL, prec, out, cap);
}
OR_API int64_t or_synth_twobody(const or_para* p, or_synth* S, int prec, or_scat* out, int64_t cap) {
    return twobody_common(p, or_synth_h2, NULL, NULL, S, NULL, NULL, prec, out, cap);
}

/* scat * mbs_in (EDCore/src/multiplication.jl:19-33): returns 1 and writes (amp, out state)
 * when the term maps the state, else 0. */
OR_API int or_scat_apply(const or_scat* sc, uint64_t st, double* re, double* im, uint64_t* out_state) {
    if ((st & sc->in) != sc->in) return 0;
    if (sc->in == sc->out) { *re = sc->re; *im = sc->im; *out_state = st; return 1; }
    uint64_t mid = st & ~sc->in;
    if ((mid & sc->out) != 0) return 0;
    int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
    *re = sign * sc->re; *im = sign * sc->im; *out_state = mid | sc->out;
    return 1;
}
/* mbs_out * scat (EDCore/src/multiplication.jl:55-69) */
OR_API int or_scat_apply_right(const or_scat* sc, uint64_t st, double* re, double* im, uint64_t* in_state) {
    if ((st & sc->out) != sc->out) return 0;
    if (sc->in == sc->out) { *re = sc->re; *im = sc->im; *in_state = st; return 1; }
    uint64_t mid = st & ~sc->out;
    if ((mid & sc->in) != 0) return 0;
    int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
    *re = sign * sc->re; *im = sign * sc->im; *in_state = mid | sc->in;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* CPU matrix-free map y = H x: MomentumED/src/method/linear_map.jl:100-118  */
/* with mbs_out * scat from EDCore/src/multiplication.jl:55-69 and the       */
/* searchsortedfirst/index_fit lookup of hilbert_subspace.jl:67-72.           */
/* Complex vectors are interleaved (re, im).                                 */
/* ------------------------------------------------------------------------ */
static inline int64_t searchsortedfirst(const uint64_t* a, int64_t n, uint64_t v) {
    int64_t lo = 0, hi = n;     /* first index with a[i] >= v (0-based); n if none */
    while (lo < hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

OR_API void or_matvec_c128(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat,
                           const double* x, double* y, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < N; ++i) {
        uint64_t st = basis[i];
        double yr = 0.0, yi = 0.0;
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->out) != sc->out) continue;
            double ar, ai;
            uint64_t tgt;
            if (sc->in == sc->out) { ar = sc->re; ai = sc->im; tgt = st; }
            else {
                uint64_t mid = st & ~sc->out;
                if ((mid & sc->in) != 0) continue;
                tgt = mid | sc->in;
                int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
                ar = sign * sc->re; ai = sign * sc->im;
            }
            if (ar == 0.0 && ai == 0.0) continue;
            int64_t j = searchsortedfirst(basis, N, tgt);
            if (j < N && basis[j] == tgt) {
                double pr, pi;
                cmul(ar, ai, x[2 * j], x[2 * j + 1], &pr, &pi);
                yr = yr + pr; yi = yi + pi;
            }
        }
        y[2 * i] = yr; y[2 * i + 1] = yi;
    }
}

OR_API void or_matvec_c64(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat,
                          const float* x, float* y, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < N; ++i) {
        uint64_t st = basis[i];
        float yr = 0.0f, yi = 0.0f;
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->out) != sc->out) continue;
            float ar, ai;
            uint64_t tgt;
            if (sc->in == sc->out) { ar = (float)sc->re; ai = (float)sc->im; tgt = st; }
            else {
                uint64_t mid = st & ~sc->out;
                if ((mid & sc->in) != 0) continue;
                tgt = mid | sc->in;
                float sign = (float)(1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1));
                ar = sign * (float)sc->re; ai = sign * (float)sc->im;
            }
            if (ar == 0.0f && ai == 0.0f) continue;
            int64_t j = searchsortedfirst(basis, N, tgt);
            if (j < N && basis[j] == tgt) {
                float pr, pi;
                cmulf(ar, ai, x[2 * j], x[2 * j + 1], &pr, &pi);
                yr = yr + pr; yi = yi + pi;
            }
        }
        y[2 * i] = yr; y[2 * i + 1] = yi;
    }
}

/* The same map evaluated on selected rows only (spot checks of large sectors). */
OR_API void or_matvec_rows_c128(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat,
                                const double* x, const int64_t* rows, int64_t nrows, double* y, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[r];
        uint64_t st = basis[i];
        double yr = 0.0, yi = 0.0;
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->out) != sc->out) continue;
            double ar, ai;
            uint64_t tgt;
            if (sc->in == sc->out) { ar = sc->re; ai = sc->im; tgt = st; }
            else {
                uint64_t mid = st & ~sc->out;
                if ((mid & sc->in) != 0) continue;
                tgt = mid | sc->in;
                int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
                ar = sign * sc->re; ai = sign * sc->im;
            }
            int64_t j = searchsortedfirst(basis, N, tgt);
            if (j < N && basis[j] == tgt) {
                double pr, pi;
                cmul(ar, ai, x[2 * j], x[2 * j + 1], &pr, &pi);
                yr = yr + pr; yi = yi + pi;
            }
        }
        y[2 * r] = yr; y[2 * r + 1] = yi;
    }
}

/* Dense H[i][j] = <i|H|j> (row-major, interleaved complex) for small cross-checks. */
OR_API void or_dense_hamiltonian(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat, double* H) {
    memset(H, 0, (size_t)N * N * 16);
    for (int64_t i = 0; i < N; ++i) {
        uint64_t st = basis[i];
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->out) != sc->out) continue;
            double ar, ai; uint64_t tgt;
            if (sc->in == sc->out) { ar = sc->re; ai = sc->im; tgt = st; }
            else {
                uint64_t mid = st & ~sc->out;
                if ((mid & sc->in) != 0) continue;
                tgt = mid | sc->in;
                int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
                ar = sign * sc->re; ai = sign * sc->im;
            }
            int64_t j = searchsortedfirst(basis, N, tgt);
            if (j < N && basis[j] == tgt) {
                H[2 * (i * N + j)] += ar;
                H[2 * (i * N + j) + 1] += ai;
            }
        }
    }
}

/* The sparse method's matrix: ED_HamiltonianMatrix_threaded_CSCdirect
 * (MomentumED/src/method/sparse_matrix.jl:64-190) with the Hermitian-completed list
 * (the else branch, 117-124): column j is the input state basis[j]; every term with
 * in within it gives (scat * mbs_in, multiplication.jl:55-69) an output state, dropped
 * when index_fit fails (hilbert_subspace.jl:67-72) or the amplitude is zero; the column's
 * (row, value) pairs are sorted by row and duplicates summed (141-156).  0-based CSC:
 * colptr[N + 1]; rowval / nzval (interleaved complex) hold at most cap entries.  Returns
 * the entries (more than cap: only the count is exact). */
OR_API int64_t or_sparse_csc(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat,
                             int64_t* colptr, int64_t* rowval, double* nzval, int64_t cap) {
    typedef struct { int64_t i; double re, im; } entry;
    entry* buf = (entry*)malloc((size_t)(nscat > 0 ? nscat : 1) * sizeof(entry));
    int64_t nnz = 0;
    colptr[0] = 0;
    for (int64_t j = 0; j < N; ++j) {
        const uint64_t st = basis[j];
        int64_t nb = 0;
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->in) != sc->in) continue;
            uint64_t tgt;
            double re, im;
            if (sc->in == sc->out) { tgt = st; re = sc->re; im = sc->im; }
            else {
                uint64_t mid = st & ~sc->in;
                if ((mid & sc->out) != 0) continue;
                tgt = mid | sc->out;
                int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
                re = sign * sc->re; im = sign * sc->im;
            }
            if (re == 0.0 && im == 0.0) continue;
            int64_t i = searchsortedfirst(basis, N, tgt);
            if (i >= N || basis[i] != tgt) continue;
            buf[nb].i = i; buf[nb].re = re; buf[nb].im = im;
            ++nb;
        }
        /* a stable sort keeps the list order among equal rows, so the sums below are formed
         * in the same order as the reference's accumulation */
        for (int64_t a = 1; a < nb; ++a) {
            entry e = buf[a];
            int64_t b = a - 1;
            while (b >= 0 && buf[b].i > e.i) { buf[b + 1] = buf[b]; --b; }
            buf[b + 1] = e;
        }
        int64_t k = 0;
        while (k < nb) {
            int64_t i = buf[k].i;
            double re = buf[k].re, im = buf[k].im;
            int64_t q = k + 1;
            while (q < nb && buf[q].i == i) { re += buf[q].re; im += buf[q].im; ++q; }
            if (nnz < cap) { rowval[nnz] = i; nzval[2 * nnz] = re; nzval[2 * nnz + 1] = im; }
            ++nnz;
            k = q;
        }
        colptr[j + 1] = nnz;
    }
    free(buf);
    return nnz;
}

/* <bra| op |ket>: mul_add_bracket / mul_add_bracket_scatlist (EDCore/src/multiplication.jl:153-190)
 * over a term list; with upper != 0 every off-diagonal term also adds its conjugate back-scatter
 * (upper_hermitian).  bra lives on bra_basis, ket on ket_basis (sorted lists); targets outside the
 * bra space are dropped (index_fit).  Vectors are interleaved complex. */
OR_API void or_bracket(const uint64_t* bra_basis, int64_t nbra, const double* bra, const uint64_t* ket_basis,
                       int64_t nket, const double* ket, const or_scat* list, int64_t nscat, int upper,
                       double* out) {
    double sr = 0.0, si = 0.0;
    for (int64_t s = 0; s < nscat; ++s) {
        const or_scat* sc = &list[s];
        double br = 0.0, bi = 0.0;
        for (int64_t j = 0; j < nket; ++j) {
            const uint64_t st = ket_basis[j];
            if ((st & sc->in) != sc->in) continue;
            uint64_t tgt;
            double ar, ai;
            if (sc->in == sc->out) { tgt = st; ar = sc->re; ai = sc->im; }
            else {
                uint64_t mid = st & ~sc->in;
                if ((mid & sc->out) != 0) continue;
                tgt = mid | sc->out;
                int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
                ar = sign * sc->re; ai = sign * sc->im;
            }
            if (ar == 0.0 && ai == 0.0) continue;
            int64_t i = searchsortedfirst(bra_basis, nbra, tgt);
            if (i >= nbra || bra_basis[i] != tgt) continue;
            /* conj(bra[i]) * amp * ket[j] */
            double kr = ket[2 * j], ki = ket[2 * j + 1], pr = ar * kr - ai * ki, pi = ar * ki + ai * kr;
            double cr = bra[2 * i], ci = -bra[2 * i + 1];
            br += cr * pr - ci * pi;
            bi += cr * pi + ci * pr;
            if (upper && i != j) {
                /* conj(bra[j]) * conj(amp) * ket[i] (the same space for bra and ket) */
                double kr2 = ket[2 * i], ki2 = ket[2 * i + 1];
                double qr = ar * kr2 + ai * ki2, qi = ar * ki2 - ai * kr2;
                double dr = bra[2 * j], di = -bra[2 * j + 1];
                br += dr * qr - di * qi;
                bi += dr * qi + di * qr;
            }
        }
        sr += br;
        si += bi;
    }
    out[0] = sr;
    out[1] = si;
}

/* PES_1rdm (MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33): the one-body
 * reduced density matrix rdm[i][j] = <psi| c+_i c_j |psi> over orbitals 1..bits, computed for
 * i <= j (sign from scat_occ_number of the intermediate state at i and j) and completed by
 * rdm[i][j] = conj(rdm[j][i]).  rdm: [bits][bits] interleaved complex, row-major. */
OR_API void or_rdm1(const uint64_t* basis, int64_t N, const double* psi, int bits, double* rdm) {
    memset(rdm, 0, (size_t)bits * bits * 16);
    for (int i = 1; i <= bits; ++i)
        for (int j = i; j <= bits; ++j) {
            double sr = 0.0, si = 0.0;
            for (int64_t x = 0; x < N; ++x) {
                uint64_t in = basis[x];
                uint64_t bj = jl_one_shl(j - 1), bi = jl_one_shl(i - 1);
                if ((in & bj) == 0) continue;
                uint64_t mid = in & ~bj;
                if (mid & bi) continue;
                uint64_t out = mid | bi;
                int64_t y = searchsortedfirst(basis, N, out);
                if (y >= N || basis[y] != out) continue;
                int par = or_scat_occ_number_1(mid, i, bits) + or_scat_occ_number_1(mid, j, bits);
                /* conj(psi[y]) * psi[x] */
                double pr = psi[2 * y] * psi[2 * x] + psi[2 * y + 1] * psi[2 * x + 1];
                double pi = psi[2 * y] * psi[2 * x + 1] - psi[2 * y + 1] * psi[2 * x];
                if (par & 1) { sr -= pr; si -= pi; } else { sr += pr; si += pi; }
            }
            rdm[2 * ((size_t)(i - 1) * bits + (j - 1))] = sr;
            rdm[2 * ((size_t)(i - 1) * bits + (j - 1)) + 1] = si;
        }
    for (int i = 1; i <= bits; ++i)
        for (int j = 1; j < i; ++j) {
            rdm[2 * ((size_t)(i - 1) * bits + (j - 1))] = rdm[2 * ((size_t)(j - 1) * bits + (i - 1))];
            rdm[2 * ((size_t)(i - 1) * bits + (j - 1)) + 1] = -rdm[2 * ((size_t)(j - 1) * bits + (i - 1)) + 1];
        }
}

/* ED_step_inner_prod (MomentumED/src/analysis/manybody_quantum_geometry.jl:48-94): for g vectors
 * psi_f[j], psi_i[k] on one basis, out[j][k] = sum_x conj(psi_f[j][x]) psi_i[k][x] * prod of
 * orb[o] over the occupied orbitals o of basis[x] (ascending, occ_list).  Vectors [g][N],
 * orb [norb], out [g][g], all interleaved complex. */
OR_API void or_step_inner_prod(const uint64_t* basis, int64_t N, const double* psi_f, const double* psi_i, int g,
                               const double* orb, int norb, double* out) {
    memset(out, 0, (size_t)g * g * 16);
    for (int64_t x = 0; x < N; ++x) {
        double pr = 1.0, pi = 0.0;
        for (int o = 0; o < norb; ++o) {
            if (!((basis[x] >> o) & 1ULL)) continue;
            double r, i;
            cmul(pr, pi, orb[2 * o], orb[2 * o + 1], &r, &i);
            pr = r; pi = i;
        }
        for (int j = 0; j < g; ++j)
            for (int k = 0; k < g; ++k) {
                double fr = psi_f[2 * ((size_t)j * N + x)], fi = -psi_f[2 * ((size_t)j * N + x) + 1];
                double ir = psi_i[2 * ((size_t)k * N + x)], ii = psi_i[2 * ((size_t)k * N + x) + 1];
                double cr, ci, vr, vi;
                cmul(fr, fi, ir, ii, &cr, &ci);
                cmul(cr, ci, pr, pi, &vr, &vi);
                out[2 * ((size_t)j * g + k)] += vr;
                out[2 * ((size_t)j * g + k) + 1] += vi;
            }
    }
}

/* <bra| op2 op1 |ket> (mul_add_bracket with two Scatters, EDCore/src/multiplication.jl:174-190,
 * summed over both lists, 215-222): amp, out = scat2 * (scat1 * ket state) with the intermediate
 * state unrestricted; the final state must lie in the bra space. */
static int scat_fwd(const or_scat* sc, uint64_t st, uint64_t* out, double* ar, double* ai) {
    if ((st & sc->in) != sc->in) return 0;
    if (sc->in == sc->out) { *out = st; *ar = sc->re; *ai = sc->im; return 1; }
    uint64_t mid = st & ~sc->in;
    if ((mid & sc->out) != 0) return 0;
    *out = mid | sc->out;
    int sign = 1 - 2 * (__builtin_popcountll(mid & sc->pm) & 1);
    *ar = sign * sc->re; *ai = sign * sc->im;
    return 1;
}

OR_API void or_bracket2(const uint64_t* bra_basis, int64_t nbra, const double* bra, const uint64_t* ket_basis,
                        int64_t nket, const double* ket, const or_scat* l2, int64_t n2, const or_scat* l1,
                        int64_t n1, double* out) {
    double sr = 0.0, si = 0.0;
    for (int64_t a = 0; a < n2; ++a)
        for (int64_t b = 0; b < n1; ++b)
            for (int64_t j = 0; j < nket; ++j) {
                uint64_t m, o;
                double r1, i1, r2, i2;
                if (!scat_fwd(&l1[b], ket_basis[j], &m, &r1, &i1)) continue;
                if (!scat_fwd(&l2[a], m, &o, &r2, &i2)) continue;
                double ar, ai;
                cmul(r2, i2, r1, i1, &ar, &ai);
                if (ar == 0.0 && ai == 0.0) continue;
                int64_t i = searchsortedfirst(bra_basis, nbra, o);
                if (i >= nbra || bra_basis[i] != o) continue;
                double pr, pi, qr, qi;
                cmul(ar, ai, ket[2 * j], ket[2 * j + 1], &pr, &pi);
                cmul(bra[2 * i], -bra[2 * i + 1], pr, pi, &qr, &qi);
                sr += qr;
                si += qi;
            }
    out[0] = sr;
    out[1] = si;
}

/* Exact nonzero count of the gather (row, term) hits, the nnz of the roofline formula. */
OR_API int64_t or_count_hits(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int64_t total = 0;
    #pragma omp parallel for schedule(dynamic, 256) reduction(+:total)
    for (int64_t i = 0; i < N; ++i) {
        uint64_t st = basis[i];
        for (int64_t s = 0; s < nscat; ++s) {
            const or_scat* sc = &list[s];
            if ((st & sc->out) != sc->out) continue;
            uint64_t tgt = st;
            if (sc->in != sc->out) {
                uint64_t mid = st & ~sc->out;
                if ((mid & sc->in) != 0) continue;
                tgt = mid | sc->in;
            }
            int64_t j = searchsortedfirst(basis, N, tgt);
            if (j < N && basis[j] == tgt) total += 1;
        }
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* Dense real symmetric eigensolver (cyclic Jacobi), ascending eigenvalues.  */
/* A is n x n row-major (destroyed); V receives eigenvectors as columns.     */
/* ------------------------------------------------------------------------ */
OR_API void or_symeig(int n, double* A, double* w, double* V) {
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) V[i * n + j] = (i == j);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) {
            tot += A[i * n + j] * A[i * n + j];
            if (i != j) off += A[i * n + j] * A[i * n + j];
        }
        if (off <= 1e-32 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
    /* sort ascending */
    for (int i = 0; i < n; ++i) {
        int mi = i;
        for (int j = i + 1; j < n; ++j) if (w[j] < w[mi]) mi = j;
        if (mi != i) {
            double t = w[i]; w[i] = w[mi]; w[mi] = t;
            for (int k = 0; k < n; ++k) { double u = V[k * n + i]; V[k * n + i] = V[k * n + mi]; V[k * n + mi] = u; }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Thick-restart (Krylov-Schur) Lanczos, FP64, full reorthogonalisation      */
/* (classical Gram-Schmidt, two passes).  Restates the algorithm KrylovKit's  */
/* eigsolve(H, x0, howmany, :SR; ishermitian=true) runs for                   */
/* krylov_map_solve (linear_map.jl:179-191): krylovdim, tol on the residual   */
/* norm |beta * last component|, maxiter restarts, keep (3m + 2 nconv)/5.     */
/* ------------------------------------------------------------------------ */
typedef struct { int32_t converged, restarts; int64_t matvecs; } or_info;

static double cdot_re_im(int64_t N, const double* a, const double* b, double* im_out) {
    double sr = 0.0, si = 0.0;
    #pragma omp parallel for reduction(+:sr,si) schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        double ar = a[2 * i], ai = a[2 * i + 1], br = b[2 * i], bi = b[2 * i + 1];
        sr += ar * br + ai * bi;   /* conj(a) * b */
        si += ar * bi - ai * br;
    }
    *im_out = si;
    return sr;
}
static double cnorm(int64_t N, const double* a) {
    double s = 0.0;
    #pragma omp parallel for reduction(+:s) schedule(static)
    for (int64_t i = 0; i < 2 * N; ++i) s += a[i] * a[i];
    return sqrt(s);
}

OR_API int or_eigsolve(const uint64_t* basis, int64_t N, const or_scat* list, int64_t nscat,
                       int nev, int krylovdim, double tol, int maxiter, const double* vec0, uint64_t seed,
                       int nthreads, double* vals, double* vecs, double* resid, or_info* info) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (N < 1 || nev < 1) return -1;
    if (nev > N) nev = (int)N;
    int m = krylovdim;
    if (m > N) m = (int)N;
    if (m < nev + 1 && m < N) m = nev + 1 < N ? nev + 1 : (int)N;
    double* V = (double*)malloc((size_t)(m + 1) * N * 16);
    double* w = (double*)malloc((size_t)N * 16);
    double* T = (double*)calloc((size_t)m * m, 8);
    double* A = (double*)malloc((size_t)m * m * 8);
    double* U = (double*)malloc((size_t)m * m * 8);
    double* th = (double*)malloc((size_t)m * 8);
    double* c = (double*)malloc((size_t)(m + 1) * 16);
    double* Vn = NULL;
    if (!V || !w || !T || !A || !U || !th || !c) return -2;
    uint64_t st = seed;
    if (vec0) memcpy(V, vec0, (size_t)N * 16);
    else for (int64_t i = 0; i < 2 * N; ++i) V[i] = u01(&st);
    double nrm = cnorm(N, V);
    for (int64_t i = 0; i < 2 * N; ++i) V[i] /= nrm;
    int k = 0, restarts = 0, nconv = 0;
    int64_t matvecs = 0;
    double beta_last = 0.0;
    int mcur = m;
    for (;;) {
        int j;
        mcur = m;
        for (j = k; j < m; ++j) {
            double* vj = V + (size_t)j * 2 * N;
            or_matvec_c128(basis, N, list, nscat, vj, w, nthreads);
            ++matvecs;
            double alpha = 0.0;
            for (int pass = 0; pass < 2; ++pass) {
                for (int i = 0; i <= j; ++i) {
                    double ci;
                    double cr = cdot_re_im(N, V + (size_t)i * 2 * N, w, &ci);
                    c[2 * i] = cr; c[2 * i + 1] = ci;
                }
                #pragma omp parallel for schedule(static)
                for (int64_t e = 0; e < N; ++e) {
                    double sr = 0.0, si = 0.0;
                    for (int i = 0; i <= j; ++i) {
                        const double* vi = V + (size_t)i * 2 * N;
                        sr += c[2 * i] * vi[2 * e] - c[2 * i + 1] * vi[2 * e + 1];
                        si += c[2 * i] * vi[2 * e + 1] + c[2 * i + 1] * vi[2 * e];
                    }
                    w[2 * e] -= sr; w[2 * e + 1] -= si;
                }
                alpha += c[2 * j];
            }
            T[j * m + j] = alpha;
            double beta = cnorm(N, w);
            if (j + 1 < m) { T[j * m + j + 1] = beta; T[(j + 1) * m + j] = beta; }
            beta_last = beta;
            double* vn = V + (size_t)(j + 1) * 2 * N;
            if (beta <= 1e-14 * (fabs(alpha) + 1.0)) {
                /* invariant subspace: restart direction is a fresh random vector orthogonal to V */
                if (j + 1 >= N) { mcur = j + 1; beta_last = 0.0; break; }
                for (int64_t i = 0; i < 2 * N; ++i) vn[i] = u01(&st) - 0.5;
                for (int pass = 0; pass < 2; ++pass)
                    for (int i = 0; i <= j; ++i) {
                        double ci;
                        double cr = cdot_re_im(N, V + (size_t)i * 2 * N, vn, &ci);
                        const double* vi = V + (size_t)i * 2 * N;
                        for (int64_t e = 0; e < N; ++e) {
                            vn[2 * e] -= cr * vi[2 * e] - ci * vi[2 * e + 1];
                            vn[2 * e + 1] -= cr * vi[2 * e + 1] + ci * vi[2 * e];
                        }
                    }
                double nn = cnorm(N, vn);
                for (int64_t i = 0; i < 2 * N; ++i) vn[i] /= nn;
                if (j + 1 < m) { T[j * m + j + 1] = 0.0; T[(j + 1) * m + j] = 0.0; }
                beta_last = 0.0;
            } else {
                for (int64_t i = 0; i < 2 * N; ++i) vn[i] = w[i] / beta;
            }
        }
        /* Rayleigh-Ritz on the projected matrix */
        int mm = mcur;
        for (int a = 0; a < mm; ++a) for (int b = 0; b < mm; ++b) A[a * mm + b] = T[a * m + b];
        or_symeig(mm, A, th, U);
        nconv = 0;
        while (nconv < nev && nconv < mm && fabs(beta_last * U[(mm - 1) * mm + nconv]) <= tol) ++nconv;
        if (nconv >= nev || restarts >= maxiter || mm < m) {
            int nout = nev < mm ? nev : mm;
            for (int i = 0; i < nout; ++i) {
                vals[i] = th[i];
                if (resid) resid[i] = fabs(beta_last * U[(mm - 1) * mm + i]);
            }
            if (vecs) {
                #pragma omp parallel for schedule(static)
                for (int64_t e = 0; e < N; ++e)
                    for (int i = 0; i < nout; ++i) {
                        double sr = 0.0, si = 0.0;
                        for (int a = 0; a < mm; ++a) {
                            const double* va = V + (size_t)a * 2 * N;
                            sr += U[a * mm + i] * va[2 * e];
                            si += U[a * mm + i] * va[2 * e + 1];
                        }
                        vecs[2 * ((size_t)i * N + e)] = sr;
                        vecs[2 * ((size_t)i * N + e) + 1] = si;
                    }
            }
            if (info) { info->converged = nconv; info->restarts = restarts; info->matvecs = matvecs; }
            break;
        }
        int keep = (3 * m + 2 * nconv) / 5;
        if (keep < nev) keep = nev;
        if (keep > m - 2) keep = m - 2;
        if (keep < 1) keep = 1;
        if (!Vn) Vn = (double*)malloc((size_t)keep * N * 16 + 16);
        else Vn = (double*)realloc(Vn, (size_t)keep * N * 16 + 16);
        #pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < N; ++e)
            for (int i = 0; i < keep; ++i) {
                double sr = 0.0, si = 0.0;
                for (int a = 0; a < m; ++a) {
                    const double* va = V + (size_t)a * 2 * N;
                    sr += U[a * m + i] * va[2 * e];
                    si += U[a * m + i] * va[2 * e + 1];
                }
                Vn[2 * ((size_t)i * N + e)] = sr;
                Vn[2 * ((size_t)i * N + e) + 1] = si;
            }
        memcpy(V + (size_t)keep * 2 * N, V + (size_t)m * 2 * N, (size_t)N * 16);
        memcpy(V, Vn, (size_t)keep * N * 16);
        memset(T, 0, (size_t)m * m * 8);
        for (int i = 0; i < keep; ++i) {
            T[i * m + i] = th[i];
            double s = beta_last * U[(m - 1) * m + i];
            T[i * m + keep] = s; T[keep * m + i] = s;
        }
        k = keep;
        ++restarts;
    }
    free(V); free(w); free(T); free(A); free(U); free(th); free(c); free(Vn);
    return 0;
}
