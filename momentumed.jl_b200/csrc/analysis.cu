// Analysis of eigenvectors on the device: the one-body reduced density matrix and the
// many-body connection step of the quantum-geometry analysis.
//
// Reference: PES_1rdm (MomentumED/src/analysis/particle_reduced_density_matrix.jl:4-33):
// rdm[i][j] = <psi| c+_i c_j |psi> for i <= j, summed over basis states x_in with j occupied,
// mid = x_in - j, i empty in mid (or i = j), x_out = mid + i found in the subspace (index_fit),
// sign (-1)^(scat_occ_number(mid, i) + scat_occ_number(mid, j)) where scat_occ_number counts
// the occupied orbitals above the given one; then rdm[i][j] = conj(rdm[j][i]) for i > j.
//
// One thread per basis state walks its occupied orbitals j and the orbitals i <= j; targets are
// looked up with key checks (c+_i c_j usually leaves a momentum sector).  A block accumulates its
// norb x norb matrix in shared memory; the host adds the blocks' matrices in block order.
#include "candidates.cuh"

namespace momed {

namespace {

constexpr int kRdmThreads = 256;

__global__ void __launch_bounds__(kRdmThreads)
k_rdm1(IndexView iv, const double2* __restrict__ psi, int norb, double2* __restrict__ partial) {
    extern __shared__ double2 acc[];                  // [norb * norb]
    __shared__ SharedTables sh;
    const int nn = norb * norb;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) acc[e] = make_double2(0.0, 0.0);
    stage_tables(sh, iv);                             // ends with __syncthreads
    const uint64_t omask = norb >= 64 ? ~0ull : ((1ull << norb) - 1ull);
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < iv.n; x += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t s = __ldg(iv.basis + x);
        const double2 pin = __ldg(psi + x);
        uint64_t rem = s & omask;
        while (rem) {
            const int j = __ffsll((long long)rem) - 1;
            rem &= rem - 1ull;
            const uint64_t mid = s & ~(1ull << j);
            const uint64_t above_j = j >= 63 ? 0ull : (~0ull << (j + 1));
            for (int i = 0; i <= j; ++i) {
                if (i != j && ((mid >> i) & 1ull)) continue;
                int64_t y = x;
                if (i != j) {
                    y = lookup_index(iv, mid | (1ull << i), sh.base_hi, sh.base_lo, sh.binom);
                    if (y < 0) continue;
                }
                const uint64_t above_i = i >= 63 ? 0ull : (~0ull << (i + 1));
                const bool neg = ((__popcll(mid & above_i) + __popcll(mid & above_j)) & 1) != 0;
                const double2 pout = __ldg(psi + y);
                double vr = pout.x * pin.x + pout.y * pin.y;      // conj(psi[y]) * psi[x]
                double vi = pout.x * pin.y - pout.y * pin.x;
                if (neg) { vr = -vr; vi = -vi; }
                atomicAdd(&acc[i * norb + j].x, vr);
                atomicAdd(&acc[i * norb + j].y, vi);
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nn; e += blockDim.x) partial[(int64_t)blockIdx.x * nn + e] = acc[e];
}

// ED_step_inner_prod (MomentumED/src/analysis/manybody_quantum_geometry.jl:48-94): thread per
// basis state; the product of the orbital overlaps over its occupied orbitals (ascending, as
// occ_list gives them), then conj(psi_f[j][x]) psi_i[k][x] times that product for every (j, k),
// accumulated per block in shared memory (g <= 32).
__global__ void __launch_bounds__(kRdmThreads)
k_step_inner(const uint64_t* __restrict__ basis, int64_t n, const double2* __restrict__ psi_f,
             const double2* __restrict__ psi_i, int g, const double2* __restrict__ orb, int norb,
             double2* __restrict__ partial) {
    extern __shared__ double2 acc[];                  // [g * g]
    __shared__ double2 s_orb[64];
    const int gg = g * g;
    for (int e = threadIdx.x; e < gg; e += blockDim.x) acc[e] = make_double2(0.0, 0.0);
    if (threadIdx.x < 64) s_orb[threadIdx.x] = threadIdx.x < norb ? orb[threadIdx.x] : make_double2(1.0, 0.0);
    __syncthreads();
    const uint64_t omask = norb >= 64 ? ~0ull : ((1ull << norb) - 1ull);
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        uint64_t rem = __ldg(basis + x) & omask;
        double pr = 1.0, pi = 0.0;
        while (rem) {
            const int o = __ffsll((long long)rem) - 1;
            rem &= rem - 1ull;
            const double2 w = s_orb[o];
            const double r = pr * w.x - pi * w.y, i = pr * w.y + pi * w.x;
            pr = r;
            pi = i;
        }
        for (int j = 0; j < g; ++j) {
            const double2 f = __ldg(psi_f + (int64_t)j * n + x);
            for (int k = 0; k < g; ++k) {
                const double2 v = __ldg(psi_i + (int64_t)k * n + x);
                const double cr = f.x * v.x + f.y * v.y, ci = f.x * v.y - f.y * v.x;   // conj(f) * v
                atomicAdd(&acc[j * g + k].x, cr * pr - ci * pi);
                atomicAdd(&acc[j * g + k].y, cr * pi + ci * pr);
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < gg; e += blockDim.x) partial[(int64_t)blockIdx.x * gg + e] = acc[e];
}

}  // namespace

void step_inner_prod(momed_handle* h, const double* psi_f, const double* psi_i, int g, const double* orb, int norb,
                     double* out) {
    MOMED_REQUIRE(g >= 1 && g <= 32, MOMED_EINVAL, "g must be in [1, 32]");
    MOMED_REQUIRE(norb >= 1 && norb <= 64, MOMED_EINVAL, "norb must be in [1, 64]");
    MOMED_REQUIRE(!h->sparse_only && h->n > 0, MOMED_ESTATE, "set a basis first (momed_set_basis)");
    MOMED_REQUIRE(norb == 64 || (h->basis_or >> norb) == 0, MOMED_EINVAL, "basis states use orbitals beyond norb");
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    DevBuf<double2> fd, id, od, part;
    fd.resize((size_t)g * n);
    id.resize((size_t)g * n);
    od.resize(norb);
    MOMED_CUDA_TRY(cudaMemcpyAsync(fd.p, psi_f, (size_t)g * n * 16, cudaMemcpyHostToDevice, st));
    MOMED_CUDA_TRY(cudaMemcpyAsync(id.p, psi_i, (size_t)g * n * 16, cudaMemcpyHostToDevice, st));
    MOMED_CUDA_TRY(cudaMemcpyAsync(od.p, orb, (size_t)norb * 16, cudaMemcpyHostToDevice, st));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kRdmThreads - 1) / kRdmThreads, (int64_t)sms * 2));
    const int gg = g * g;
    part.resize((size_t)grid * gg);
    k_step_inner<<<grid, kRdmThreads, (size_t)gg * sizeof(double2), st>>>(h->basis.p, n, fd.p, id.p, g, od.p, norb,
                                                                          part.p);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    std::vector<double2> hp((size_t)grid * gg);
    MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 16, cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    for (int e = 0; e < gg; ++e) {
        double re = 0.0, im = 0.0;
        for (int b = 0; b < grid; ++b) {
            re += hp[(size_t)b * gg + e].x;
            im += hp[(size_t)b * gg + e].y;
        }
        out[2 * e] = re;
        out[2 * e + 1] = im;
    }
}

void rdm1(momed_handle* h, const double* psi, int norb, double* rdm) {
    MOMED_REQUIRE(norb >= 1 && norb <= 64, MOMED_EINVAL, "norb must be in [1, 64]");
    MOMED_REQUIRE(!h->sparse_only && h->n > 0, MOMED_ESTATE, "set a basis first (momed_set_basis)");
    MOMED_REQUIRE(norb == 64 || (h->basis_or >> norb) == 0, MOMED_EINVAL, "basis states use orbitals beyond norb");
    if (h->index_dirty || (h->op_mask_or & ~h->index_bits)) {
        h->index_bits = h->basis_or | h->op_mask_or;
        build_index(h);
        h->index_dirty = false;
        h->op_validated = false;
    }
    IndexView iv = index_view(h);
    if (iv.mode == INDEX_RANKED) iv.mode = INDEX_CHECKED;     // targets leave the sector: compare keys
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    DevBuf<double2> pd, part;
    pd.resize(n);
    MOMED_CUDA_TRY(cudaMemcpyAsync(pd.p, psi, n * 16, cudaMemcpyHostToDevice, st));
    const int nn = norb * norb;
    const size_t smem = (size_t)nn * sizeof(double2);
    constexpr size_t smem_max = 64 * 64 * sizeof(double2);
    // process-wide kernel attribute: always the largest size, so concurrent callers never lower it
    MOMED_CUDA_TRY(cudaFuncSetAttribute(k_rdm1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kRdmThreads - 1) / kRdmThreads, (int64_t)sms * 2));
    part.resize((size_t)grid * nn);
    k_rdm1<<<grid, kRdmThreads, smem, st>>>(iv, pd.p, norb, part.p);
    MOMED_CUDA_TRY(cudaGetLastError());
    note_launches(1);
    std::vector<double2> hp((size_t)grid * nn);
    MOMED_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, hp.size() * 16, cudaMemcpyDeviceToHost, st));
    MOMED_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < norb; ++i)
        for (int j = 0; j < norb; ++j) {
            double re = 0.0, im = 0.0;
            if (i <= j) {
                for (int b = 0; b < grid; ++b) {
                    re += hp[(size_t)b * nn + i * norb + j].x;
                    im += hp[(size_t)b * nn + i * norb + j].y;
                }
            }
            rdm[2 * ((size_t)i * norb + j)] = re;
            rdm[2 * ((size_t)i * norb + j) + 1] = im;
        }
    for (int i = 0; i < norb; ++i)
        for (int j = 0; j < i; ++j) {
            rdm[2 * ((size_t)i * norb + j)] = rdm[2 * ((size_t)j * norb + i)];
            rdm[2 * ((size_t)i * norb + j) + 1] = -rdm[2 * ((size_t)j * norb + i) + 1];
        }
}

}  // namespace momed
