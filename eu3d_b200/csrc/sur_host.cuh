// Host side of the learned chemistry surrogate (C ABI in include/eu3d_gpu.h):
// the training set on the device, FP64 labelling, the training loop over
// the tensor-core GEMM and the elementwise kernels of mlp.cuh with Adam,
// inference, and the coupled chemistry step of a flowfield handle.
// Included once, at the end of eu3d_gpu.cu (one translation unit).
#pragma once

#include <cuda_bf16.h>

struct eu3d_surrogate {
    int dev = 0;
    cudaStream_t st = nullptr;
    unsigned quirks = 0;
    bool spec = false;
    AdaptCfg acfg{0.02, 0.5, 4096};  // adaptive labels (nmax: the label call's cap)
    long long cap = 0, n = 0;
    double *states = nullptr;
    float *X = nullptr, *Lb = nullptr;
    // parameters (FP32 master), gradient, Adam moments, BF16 copies
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    int adam_t = 0;
    __nv_bfloat16 *W[4] = {}, *Wt[4] = {};
    float norm_h[EU3D_SUR_NORM_LEN] = {};
    SurNorm *norm_d = nullptr;
    int *err = nullptr;
    // training buffers for batch B
    int B = 0;
    float *Xb = nullptr, *Yb = nullptr, *acc = nullptr, *Z[3] = {}, *out4 = nullptr, *dH = nullptr, *dW[4] = {},
          *db[4] = {}, *loss = nullptr;
    int loss_cap = 0;
    __nv_bfloat16 *H0 = nullptr, *H0t = nullptr, *H[3] = {}, *Ht[3] = {}, *dZ4 = nullptr, *dZ4t = nullptr,
                  *dZ = nullptr, *dZt = nullptr;
    std::vector<void *> train_bufs;
    // standalone inference staging
    float *in_d = nullptr, *out_d = nullptr;
    long long io_cap = 0;
};

namespace {

const int SUR_W_IN[4] = {SUR_IN, SUR_H, SUR_H, SUR_H};
const int SUR_W_OUT[4] = {SUR_H, SUR_H, SUR_H, SUR_OUT};
constexpr int SUR_SPLITK = 256;  // batch rows per split-K block of the weight-gradient GEMMs

void sur_free_train(eu3d_surrogate *s)
{
    for (void *q : s->train_bufs) cudaFree(q);
    s->train_bufs.clear();
    s->B = 0;
}

void sur_free(eu3d_surrogate *s)
{
    sur_free_train(s);
    void *ptrs[] = {s->states, s->X, s->Lb, s->p, s->g, s->m, s->v, s->norm_d, s->err, s->loss, s->in_d, s->out_d};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    for (int l = 0; l < 4; l++) {
        if (s->W[l]) cudaFree(s->W[l]);
        if (s->Wt[l]) cudaFree(s->Wt[l]);
    }
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
}

template <class T>
int sur_alloc(eu3d_surrogate *s, T **ptr, size_t count, bool zero = true)
{
    void *q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(EU3D_ERR_NOMEM, "surrogate: device allocation failed");
    }
    if (zero) CK(cudaMemset(q, 0, count * sizeof(T)));
    s->train_bufs.push_back(q);
    *ptr = (T *)q;
    return EU3D_OK;
}

int sur_ensure_batch(eu3d_surrogate *s, int B)
{
    if (s->B == B) return EU3D_OK;
    sur_free_train(s);
    int rc;
#define SA(ptr, n) \
    if ((rc = sur_alloc(s, &(ptr), (size_t)(n)))) return rc
    SA(s->Xb, (size_t)B * SUR_IN);
    SA(s->Yb, (size_t)B * SUR_OUT);
    SA(s->acc, (size_t)B * SUR_H);
    for (int l = 0; l < 3; l++) {
        SA(s->Z[l], (size_t)B * SUR_H);
        SA(s->H[l], (size_t)B * SUR_H);
        SA(s->Ht[l], (size_t)B * SUR_H);
    }
    SA(s->out4, (size_t)B * SUR_OUT);
    SA(s->dH, (size_t)B * SUR_H);
    SA(s->H0, (size_t)B * SUR_IN);
    SA(s->H0t, (size_t)SUR_H * B);  // rows 16..127 stay zero (M padding of the dW1 GEMM)
    SA(s->dZ4, (size_t)B * SUR_OUT);
    SA(s->dZ4t, (size_t)SUR_OUT * B);
    SA(s->dZ, (size_t)B * SUR_H);
    SA(s->dZt, (size_t)SUR_H * B);
    for (int l = 0; l < 4; l++) {
        SA(s->dW[l], (size_t)SUR_H * SUR_W_OUT[l]);
        SA(s->db[l], (size_t)SUR_W_OUT[l]);
    }
#undef SA
    s->B = B;
    return EU3D_OK;
}

void sur_gemm(eu3d_surrogate *s, const __nv_bfloat16 *A, const __nv_bfloat16 *Bm, float *C, int M, int N, int K,
              bool splitk)
{
    if (splitk) {
        const int ns = (K + SUR_SPLITK - 1) / SUR_SPLITK;
        cudaMemsetAsync(C, 0, (size_t)M * N * sizeof(float), s->st);
        k_gemm_tc<<<dim3(M / 128, ns), 128, gemm_smem_bytes(), s->st>>>(A, Bm, C, M, N, K, 0, s->err, SUR_SPLITK);
    } else {
        k_gemm_tc<<<M / 128, 128, gemm_smem_bytes(), s->st>>>(A, Bm, C, M, N, K, 0, s->err, 0);
    }
}

int ew_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

// forward + loss + backward on the batch already in Xb / Yb; gradient to s->g
void sur_fwd_bwd(eu3d_surrogate *s, float *loss_slot)
{
    const int B = s->B;
    cudaStream_t st = s->st;
    const long long nh = (long long)B * SUR_H;
    const float *bias[4] = {s->p + SUR_OFF_B1, s->p + SUR_OFF_B2, s->p + SUR_OFF_B3, s->p + SUR_OFF_B4};
    k_sur_input<<<ew_blocks((long long)B * SUR_IN), 256, 0, st>>>(s->Xb, s->H0, s->H0t, B);
    const __nv_bfloat16 *in = s->H0;
    for (int l = 0; l < 3; l++) {
        sur_gemm(s, in, s->Wt[l], s->acc, B, SUR_H, SUR_W_IN[l], false);
        k_sur_fwd_act<<<ew_blocks(nh), 256, 0, st>>>(s->acc, bias[l], s->Z[l], s->H[l], s->Ht[l], B, SUR_H);
        in = s->H[l];
    }
    sur_gemm(s, in, s->Wt[3], s->acc, B, SUR_OUT, SUR_H, false);
    k_sur_loss<<<ew_blocks((long long)B * SUR_OUT), 256, 0, st>>>(s->acc, bias[3], s->Yb, s->out4, s->dZ4, s->dZ4t,
                                                                  loss_slot, B);
    // layer 4
    sur_gemm(s, s->Ht[2], s->dZ4t, s->dW[3], SUR_H, SUR_OUT, B, true);
    k_sur_colsum<<<SUR_OUT, 256, 0, st>>>(s->dZ4t, s->db[3], B);
    sur_gemm(s, s->dZ4, s->W[3], s->dH, B, SUR_H, SUR_OUT, false);
    // layers 3, 2, 1
    for (int l = 2; l >= 0; l--) {
        k_sur_bwd_act<<<ew_blocks(nh), 256, 0, st>>>(s->dH, s->Z[l], s->dZ, s->dZt, B, SUR_H);
        const __nv_bfloat16 *At = l > 0 ? s->Ht[l - 1] : s->H0t;
        sur_gemm(s, At, s->dZt, s->dW[l], SUR_H, SUR_H, B, true);
        k_sur_colsum<<<SUR_H, 256, 0, st>>>(s->dZt, s->db[l], B);
        if (l > 0) sur_gemm(s, s->dZ, s->W[l], s->dH, B, SUR_H, SUR_H, false);
    }
    k_sur_gather_grads<<<ew_blocks(SUR_NPARAM), 256, 0, st>>>(s->dW[0], s->dW[1], s->dW[2], s->dW[3], s->db[0],
                                                             s->db[1], s->db[2], s->db[3], s->g);
}

void sur_refresh(eu3d_surrogate *s)
{
    SurBf16 w;
    for (int l = 0; l < 4; l++) {
        w.W[l] = s->W[l];
        w.Wt[l] = s->Wt[l];
    }
    k_sur_refresh_bf16<<<64, 256, 0, s->st>>>(s->p, w);
}

SurWeights sur_weights(const eu3d_surrogate *s)
{
    SurWeights w;
    for (int l = 0; l < 4; l++) w.Wt[l] = s->Wt[l];
    w.p = s->p;
    return w;
}

int sur_check_err(eu3d_surrogate *s)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (e) {
        CK(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
        return fail(EU3D_ERR_CUDA, "surrogate: a tensor-core wait ran out of its bound");
    }
    return EU3D_OK;
}

int sur_ensure_io(eu3d_surrogate *s, long long n)
{
    if (s->io_cap >= n) return EU3D_OK;
    if (s->in_d) cudaFree(s->in_d);
    if (s->out_d) cudaFree(s->out_d);
    s->in_d = s->out_d = nullptr;
    s->io_cap = 0;
    CK(cudaMalloc(&s->in_d, (size_t)n * SUR_IN * sizeof(float)));
    CK(cudaMalloc(&s->out_d, (size_t)n * SUR_OUT * sizeof(float)));
    s->io_cap = n;
    return EU3D_OK;
}

int sur_grid(long long ntiles)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    return (int)std::max<long long>(1, std::min<long long>(sms, (ntiles + SUR_NG - 1) / SUR_NG));
}

int sur_set_attrs()
{
    static bool done = false;
    if (done) return EU3D_OK;
    CK(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes()));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcArray>, cudaFuncAttributeMaxDynamicSharedMemorySize, SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcField<float>>, cudaFuncAttributeMaxDynamicSharedMemorySize, SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcField<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize, SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcFieldApply<float>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcFieldApply<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcList<float>>, cudaFuncAttributeMaxDynamicSharedMemorySize, SURK_SMEM));
    CK(cudaFuncSetAttribute(k_sur_mlp<SurSrcList<double>>, cudaFuncAttributeMaxDynamicSharedMemorySize, SURK_SMEM));
    done = true;
    return EU3D_OK;
}

// ---------------------------------------------------------- coupled step
template <class P, bool SPEC>
void sur_predict_t(eu3d_handle *h, bool decoded, const SurQueue &qu)
{
    eu3d_surrogate *s = h->sur;
    const Layout &L = h->L;
    const long long n = L.interior_cells();
    P *q = (P *)h->prim;
    // [0] fallback list length, [1] its work cursor, [2] active list length;
    // an SSP-RK2 stage 2 with the gate fused in has listed the active cells
    // (and the gate's audit sample) already, from counts it set to zero
    const bool gated = h->sur_gated;
    h->sur_gated = false;
    if (!gated) cudaMemsetAsync(h->sur_count, 0, 4 * sizeof(int), h->st);
    // a new list: the balancing of the previous one is void until eu3d_sur_load
    h->sdlb_total = -1;
    h->sdlb_keep = 0;
    h->sdlb_segs = DlbGuestSegs{};
    // split step: the flux update and its decode first (Update_after_Adv),
    // unless the time scheme left the state decoded with the update in
    if (!decoded) launch_cell_t<P, SPEC>(h, M_ADV);
    SurApplyArgs a{cell_args(h), s->norm_d, h->sur_out, n, qu, h->sur_audit_stride};
    const SurSrcField<P> src{L, h->T, q, h->scal, h->sur_out, n, (L.ni + 127) / 128};
    const long long ntiles = src.ntiles();
    if (h->gate_T > 0.0) {
        // frozen-chemistry gate: the network and its apply take the listed
        // (active) cells only
        int *acount = h->sur_count + 2;
        if (!gated) {
            ProfScope ps(h, "sur_gate");
            const SurGate g{h->gate_T, (float)h->gate_y, h->gate_mask, h->gate_audit, h->sur_active, acount};
            const dim3 gg(L.nj * L.nk, (L.ni + GATE_ROW - 1) / GATE_ROW);
            k_sur_gate<P><<<gg, GATE_THREADS, 0, h->st>>>(cell_args(h), q, g, qu);
        }
        const SurSrcList<P> lsrc{L, h->T, q, h->scal, h->sur_out, h->sur_active, acount, n};
        {
            ProfScope ps(h, "sur_mlp");
            k_sur_mlp<SurSrcList<P>><<<sur_grid(lsrc.ntiles()), 128 * SUR_NG, SURK_SMEM, h->st>>>(
                sur_weights(s), s->norm_d, lsrc, lsrc.ntiles(), s->err);
        }
        {
            ProfScope ps(h, "sur_apply");
            k_sur_apply_list<P><<<(unsigned)std::max<long long>(1, (n + 127) / 128), 128, 0, h->st>>>(
                a, q, h->sur_active, acount);
        }
    } else if (h->sur_fused) {
        // network and apply in one kernel (outputs stay on chip)
        ProfScope ps(h, "sur_mlp_apply");
        SurSrcFieldApply<P> fsrc;
        static_cast<SurSrcField<P> &>(fsrc) = src;
        fsrc.ap = a;
        fsrc.q = q;
        k_sur_mlp<SurSrcFieldApply<P>><<<sur_grid(ntiles), 128 * SUR_NG, SURK_SMEM, h->st>>>(sur_weights(s), s->norm_d,
                                                                                         fsrc, ntiles, s->err);
    } else {
        {
            ProfScope ps(h, "sur_mlp");
            k_sur_mlp<SurSrcField<P>><<<sur_grid(ntiles), 128 * SUR_NG, SURK_SMEM, h->st>>>(sur_weights(s), s->norm_d,
                                                                                        src, ntiles, s->err);
        }
        ProfScope ps(h, "sur_apply");
        k_sur_apply<P><<<cell_grid(L, 128), 128, 0, h->st>>>(a, q);
    }
}

template <class P, bool SPEC>
void sur_chem_t(eu3d_handle *h, bool decoded, int half)
{
    const Layout &L = h->L;
    const long long n = L.interior_cells();
    P *q = (P *)h->prim;
    SurQueue qu{h->sur_list, h->sur_count, h->sur_audit, n, h->sur_res, h->sur_info};
    if (half & SUR_HALF_PREDICT) sur_predict_t<P, SPEC>(h, decoded, qu);
    if (half & SUR_HALF_WORK) {
        {
            ProfScope ps(h, "sur_fallback");
            k_sur_fallback<P, SPEC><<<h->nparts, 128, 0, h->st>>>(cell_args(h), q, qu);
        }
        ProfScope ps(h, "sur_fallback_finish");
        k_sur_fallback_finish<P, SPEC><<<FALLBACK_FINISH_BLOCKS, 128, 0, h->st>>>(cell_args(h), q, qu);
    }
}

template <class P, bool SPEC>
void rk2_gate_t(eu3d_handle *h)
{
    const Layout &L = h->L;
    const CellArgs a = cell_args(h);
    P *q = (P *)h->prim;
    const SurQueue qu{h->sur_list, h->sur_count, h->sur_audit, L.interior_cells(), h->sur_res, h->sur_info};
    const SurGate g{h->gate_T, (float)h->gate_y, h->gate_mask, h->gate_audit, h->sur_active, h->sur_count + 2};
    const dim3 grid = cell_grid(L, 128);
    ProfScope ps(h, "cell_rk2");
    if (sizeof(P) == 4 && h->cell_blocks == 4)
        k_rk2_gate<P, SPEC, 4><<<grid, 128, 0, h->st>>>(a, q, g, qu);
    else
        k_rk2_gate<P, SPEC, 3><<<grid, 128, 0, h->st>>>(a, q, g, qu);
}

int rk2_gate_op(eu3d_handle *h)
{
    // the new lists start empty; the stage appends the active cells and the
    // audit sample, and the surrogate step that follows keeps them
    CK(cudaMemsetAsync(h->sur_count, 0, 4 * sizeof(int), h->st));
    if (h->flux_bits == 64) {
        if (h->spec) rk2_gate_t<double, true>(h);
        else rk2_gate_t<double, false>(h);
    } else {
        if (h->spec) rk2_gate_t<float, true>(h);
        else rk2_gate_t<float, false>(h);
    }
    CK(cudaGetLastError());
    h->sur_gated = true;
    return EU3D_OK;
}

int sur_chem_op(eu3d_handle *h, bool decoded, int half)
{
    if (!h->sur) return fail(EU3D_ERR_STATE, "no surrogate attached (eu3d_set_surrogate)");
    if (h->flux_bits == 64) {
        if (h->spec) sur_chem_t<double, true>(h, decoded, half);
        else sur_chem_t<double, false>(h, decoded, half);
    } else {
        if (h->spec) sur_chem_t<float, true>(h, decoded, half);
        else sur_chem_t<float, false>(h, decoded, half);
    }
    CK(cudaGetLastError());
    return EU3D_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

int eu3d_sur_create(eu3d_handle *h, long long capacity, const double *atoms, eu3d_surrogate **out)
{
    if (!h || !atoms || !out) return fail(EU3D_ERR_ARG, "null argument");
    if (capacity < 0) return fail(EU3D_ERR_ARG, "capacity must be >= 0");
    *out = nullptr;
    CK(cudaSetDevice(h->dev));
    int rc;
    if ((rc = sur_set_attrs())) return rc;
    if ((rc = eu3d_set_elements(h, atoms))) return rc;
    eu3d_surrogate *s = new eu3d_surrogate();
    s->acfg = h->acfg;
    s->dev = h->dev;
    s->quirks = h->quirks;
    s->spec = h->spec;
    s->cap = capacity;
#define SC(call)                    \
    do {                            \
        cudaError_t e_ = (call);    \
        if (e_ != cudaSuccess) {    \
            sur_free(s);            \
            return fail(EU3D_ERR_NOMEM, std::string("surrogate: ") + cudaGetErrorString(e_)); \
        }                           \
    } while (0)
    SC(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    if (capacity > 0) {
        SC(cudaMalloc(&s->states, (size_t)capacity * 12 * sizeof(double)));
        SC(cudaMalloc(&s->X, (size_t)capacity * 12 * sizeof(float)));
        SC(cudaMalloc(&s->Lb, (size_t)capacity * 12 * sizeof(float)));
    }
    float **fp[] = {&s->p, &s->g, &s->m, &s->v};
    for (float **f : fp) {
        SC(cudaMalloc(f, SUR_NPARAM * sizeof(float)));
        SC(cudaMemset(*f, 0, SUR_NPARAM * sizeof(float)));
    }
    for (int l = 0; l < 4; l++) {
        SC(cudaMalloc(&s->W[l], (size_t)SUR_W_IN[l] * SUR_W_OUT[l] * sizeof(__nv_bfloat16)));
        SC(cudaMalloc(&s->Wt[l], (size_t)SUR_W_IN[l] * SUR_W_OUT[l] * sizeof(__nv_bfloat16)));
    }
    SC(cudaMalloc(&s->norm_d, sizeof(SurNorm)));
    SC(cudaMemset(s->norm_d, 0, sizeof(SurNorm)));
    SC(cudaMalloc(&s->err, sizeof(int)));
    SC(cudaMemset(s->err, 0, sizeof(int)));
#undef SC
    sur_refresh(s);
    *out = s;
    return EU3D_OK;
}

int eu3d_sur_destroy(eu3d_surrogate *s)
{
    if (!s) return EU3D_OK;
    cudaSetDevice(s->dev);
    cudaStreamSynchronize(s->st);
    sur_free(s);
    return EU3D_OK;
}

int eu3d_sur_reset_dataset(eu3d_surrogate *s)
{
    if (!s) return fail(EU3D_ERR_ARG, "null surrogate");
    s->n = 0;
    return EU3D_OK;
}

int eu3d_sur_add_random(eu3d_surrogate *s, long long n, const double *env, const int *species,
                        unsigned long long seed)
{
    if (!s || !env || !species) return fail(EU3D_ERR_ARG, "null argument");
    if (n < 0 || s->n + n > s->cap) return fail(EU3D_ERR_ARG, "sample count exceeds the dataset capacity");
    for (int k = 0; k < 9; k++)
        if (species[k] < 0 || species[k] >= NS) return fail(EU3D_ERR_ARG, "species index out of range");
    if (!(env[0] > 0 && env[1] >= env[0] && env[3] >= env[2] && env[5] >= env[4]))
        return fail(EU3D_ERR_ARG, "envelope bounds must be ordered, T > 0");
    CK(cudaSetDevice(s->dev));
    SurSpecies sp{species[0], species[1], species[2], species[3], species[4], species[5], species[6], species[7],
                  species[8]};
    if (n > 0)
        k_sur_random<<<(unsigned)((n + 127) / 128), 128, 0, s->st>>>(s->states, s->n, n, seed, sp, env[0], env[1],
                                                                     env[2], env[3], env[4], env[5]);
    CK(cudaGetLastError());
    s->n += n;
    return EU3D_OK;
}

int eu3d_sur_add_snapshot(eu3d_surrogate *s, eu3d_handle *src, long long n, long long stride, long long offset,
                          double jitter_T, double jitter_lnp, double lndt_lo, double lndt_hi,
                          unsigned long long seed)
{
    if (!s || !src) return fail(EU3D_ERR_ARG, "null argument");
    if (n < 0 || s->n + n > s->cap) return fail(EU3D_ERR_ARG, "sample count exceeds the dataset capacity");
    if (stride < 1 || offset < 0 || (n > 0 && offset + (n - 1) * stride >= src->L.interior_cells()))
        return fail(EU3D_ERR_ARG, "snapshot samples run past the interior cells");
    if (src->dev != s->dev) return fail(EU3D_ERR_ARG, "snapshot handle on another device");
    CK(cudaSetDevice(s->dev));
    // the snapshot is read on the surrogate's stream once the handle's queued work is done
    CK(cudaStreamSynchronize(src->st));
    if (n > 0) {
        const unsigned nb = (unsigned)((n + 127) / 128);
        if (src->flux_bits == 64)
            k_sur_snapshot<double><<<nb, 128, 0, s->st>>>(s->states, s->n, n, src->L, src->T, (const double *)src->prim,
                                                          stride, offset, seed, jitter_T, jitter_lnp, lndt_lo, lndt_hi);
        else
            k_sur_snapshot<float><<<nb, 128, 0, s->st>>>(s->states, s->n, n, src->L, src->T, (const float *)src->prim,
                                                         stride, offset, seed, jitter_T, jitter_lnp, lndt_lo, lndt_hi);
    }
    CK(cudaGetLastError());
    s->n += n;
    return EU3D_OK;
}

int eu3d_sur_label(eu3d_surrogate *s, int kind, int cap, double proj_eps, long long *n_valid)
{
    if (!s) return fail(EU3D_ERR_ARG, "null surrogate");
    if (kind != EU3D_REACT_IMEX && kind != EU3D_REACT_TRAPEZOID && kind != EU3D_REACT_ADAPTIVE)
        return fail(EU3D_ERR_ARG, "label integrator must be EU3D_REACT_ADAPTIVE, _IMEX or _TRAPEZOID");
    if (cap < 1 || cap > NCHEM_CAP) return fail(EU3D_ERR_ARG, "substep cap out of range");
    if (!(proj_eps > 0)) return fail(EU3D_ERR_ARG, "projection weight floor must be > 0");
    CK(cudaSetDevice(s->dev));
    const int k = kind == EU3D_REACT_IMEX       ? SUR_LABEL_IMEX
                  : kind == EU3D_REACT_ADAPTIVE ? SUR_LABEL_ADAPTIVE
                                                : SUR_LABEL_TRAPEZOID;
    if (s->n > 0) {
        const unsigned nb = (unsigned)((s->n + 127) / 128);
        if (s->spec)
            k_sur_label<true><<<nb, 128, 0, s->st>>>(s->states, s->n, k, s->quirks, cap, proj_eps, s->acfg, s->X,
                                                     s->Lb);
        else
            k_sur_label<false><<<nb, 128, 0, s->st>>>(s->states, s->n, k, s->quirks, cap, proj_eps, s->acfg, s->X,
                                                      s->Lb);
    }
    CK(cudaGetLastError());
    if (n_valid) {
        std::vector<float> w((size_t)s->n * 12);
        if (s->n > 0)
            CK(cudaMemcpyAsync(w.data(), s->Lb, w.size() * sizeof(float), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        long long c = 0;
        for (long long i = 0; i < s->n; i++) c += w[(size_t)i * 12 + 10] > 0.f;
        *n_valid = c;
    }
    return EU3D_OK;
}

int eu3d_sur_get_dataset(eu3d_surrogate *s, long long first, long long count, double *states, float *X, float *L)
{
    if (!s) return fail(EU3D_ERR_ARG, "null surrogate");
    if (first < 0 || count < 0 || first + count > s->n) return fail(EU3D_ERR_ARG, "range outside the dataset");
    CK(cudaSetDevice(s->dev));
    if (count > 0) {
        if (states)
            CK(cudaMemcpyAsync(states, s->states + first * 12, (size_t)count * 12 * sizeof(double),
                               cudaMemcpyDeviceToHost, s->st));
        if (X)
            CK(cudaMemcpyAsync(X, s->X + first * 12, (size_t)count * 12 * sizeof(float), cudaMemcpyDeviceToHost, s->st));
        if (L)
            CK(cudaMemcpyAsync(L, s->Lb + first * 12, (size_t)count * 12 * sizeof(float), cudaMemcpyDeviceToHost,
                               s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    return EU3D_OK;
}

int eu3d_sur_dataset_size(eu3d_surrogate *s, long long *n)
{
    if (!s || !n) return fail(EU3D_ERR_ARG, "null argument");
    *n = s->n;
    return EU3D_OK;
}

int eu3d_sur_set_norm(eu3d_surrogate *s, const float *norm)
{
    if (!s || !norm) return fail(EU3D_ERR_ARG, "null argument");
    for (int k = 0; k < SUR_NIN; k++)
        if (!(norm[SN_IN_STD + k] > 0)) return fail(EU3D_ERR_ARG, "input scales must be > 0");
    for (int k = 0; k < SUR_NOUT; k++)
        if (!(norm[SN_OUT_STD + k] > 0) || !(norm[SN_LIN + k] > 0)) return fail(EU3D_ERR_ARG, "output scales must be > 0");
    if (!(norm[SN_TR] > 0)) return fail(EU3D_ERR_ARG, "activity reference temperature must be > 0");
    CK(cudaSetDevice(s->dev));
    memcpy(s->norm_h, norm, sizeof(s->norm_h));
    CK(cudaMemcpyAsync(s->norm_d, s->norm_h, sizeof(SurNorm), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return EU3D_OK;
}

int eu3d_sur_get_norm(eu3d_surrogate *s, float *norm)
{
    if (!s || !norm) return fail(EU3D_ERR_ARG, "null argument");
    memcpy(norm, s->norm_h, sizeof(s->norm_h));
    return EU3D_OK;
}

int eu3d_sur_set_params(eu3d_surrogate *s, const float *params)
{
    if (!s || !params) return fail(EU3D_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->dev));
    CK(cudaMemcpyAsync(s->p, params, SUR_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->m, 0, SUR_NPARAM * sizeof(float), s->st));
    CK(cudaMemsetAsync(s->v, 0, SUR_NPARAM * sizeof(float), s->st));
    s->adam_t = 0;
    sur_refresh(s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->st));
    return EU3D_OK;
}

int eu3d_sur_get_params(eu3d_surrogate *s, float *params)
{
    if (!s || !params) return fail(EU3D_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->dev));
    CK(cudaMemcpyAsync(params, s->p, SUR_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return EU3D_OK;
}

int eu3d_sur_train(eu3d_surrogate *s, int steps, int batch, float lr_max, float lr_min, int warmup,
                   unsigned long long seed, float *losses)
{
    if (!s) return fail(EU3D_ERR_ARG, "null surrogate");
    if (steps < 0 || batch < 128 || batch % SUR_SPLITK != 0) return fail(EU3D_ERR_ARG, "batch must be a multiple of 256");
    if (s->n < 1) return fail(EU3D_ERR_STATE, "empty training set");
    CK(cudaSetDevice(s->dev));
    int rc;
    if ((rc = sur_ensure_batch(s, batch))) return rc;
    if (s->loss_cap < steps + 1) {
        if (s->loss) cudaFree(s->loss);
        s->loss = nullptr;
        s->loss_cap = 0;
        CK(cudaMalloc(&s->loss, (size_t)(steps + 1) * sizeof(float)));
        s->loss_cap = steps + 1;
    }
    CK(cudaMemsetAsync(s->loss, 0, (size_t)(steps + 1) * sizeof(float), s->st));
    SurNorm nrm;
    memcpy(nrm.v, s->norm_h, sizeof(nrm.v));
    for (int it = 0; it < steps; it++) {
        float lr = lr_max;
        if (it < warmup) {
            lr = lr_max * (float)(it + 1) / (float)warmup;
        } else if (steps > warmup) {
            const double f = (double)(it - warmup) / (double)(steps - warmup);
            lr = (float)(lr_min + 0.5 * (lr_max - lr_min) * (1.0 + cos(M_PI * f)));
        }
        k_sur_batch<<<(batch + 127) / 128, 128, 0, s->st>>>(s->X, s->Lb, s->n, nrm, seed, (long long)s->adam_t, batch,
                                                            s->Xb, s->Yb);
        sur_fwd_bwd(s, s->loss + it);
        s->adam_t++;
        k_sur_adam<<<ew_blocks(SUR_NPARAM), 256, 0, s->st>>>(s->p, s->g, s->m, s->v, lr, 0.9f, 0.999f, 1e-8f, s->adam_t);
        sur_refresh(s);
    }
    CK(cudaGetLastError());
    if (losses && steps > 0)
        CK(cudaMemcpyAsync(losses, s->loss, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return sur_check_err(s);
}

int eu3d_sur_loss_grad(eu3d_surrogate *s, const float *Xb, const float *Yb, int batch, float *loss, float *grad,
                       float *out)
{
    if (!s || !Xb || !Yb) return fail(EU3D_ERR_ARG, "null argument");
    if (batch < 256 || batch % SUR_SPLITK != 0) return fail(EU3D_ERR_ARG, "batch must be a multiple of 256");
    CK(cudaSetDevice(s->dev));
    int rc;
    if ((rc = sur_ensure_batch(s, batch))) return rc;
    if (s->loss_cap < 1) {
        CK(cudaMalloc(&s->loss, sizeof(float)));
        s->loss_cap = 1;
    }
    CK(cudaMemcpyAsync(s->Xb, Xb, (size_t)batch * SUR_IN * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->Yb, Yb, (size_t)batch * SUR_OUT * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->loss, 0, sizeof(float), s->st));
    sur_fwd_bwd(s, s->loss);
    CK(cudaGetLastError());
    if (loss) CK(cudaMemcpyAsync(loss, s->loss, sizeof(float), cudaMemcpyDeviceToHost, s->st));
    if (grad) CK(cudaMemcpyAsync(grad, s->g, SUR_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    if (out)
        CK(cudaMemcpyAsync(out, s->out4, (size_t)batch * SUR_OUT * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return sur_check_err(s);
}

int eu3d_sur_infer(eu3d_surrogate *s, const float *X_dev, long long n, float *out_dev, void *stream)
{
    if (!s || (n > 0 && (!X_dev || !out_dev))) return fail(EU3D_ERR_ARG, "null argument");
    if (((uintptr_t)X_dev | (uintptr_t)out_dev) & 15) return fail(EU3D_ERR_ARG, "buffers must be 16-byte aligned");
    if (n <= 0) return EU3D_OK;
    CK(cudaSetDevice(s->dev));
    const long long ntiles = (n + 127) / 128;
    SurSrcArray src{X_dev, out_dev, n};
    cudaStream_t st = stream ? (cudaStream_t)stream : s->st;
    k_sur_mlp<SurSrcArray><<<sur_grid(ntiles), 128 * SUR_NG, SURK_SMEM, st>>>(sur_weights(s), s->norm_d, src, ntiles,
                                                                             s->err);
    CK(cudaGetLastError());
    return EU3D_OK;
}

int eu3d_sur_predict(eu3d_surrogate *s, const float *X, long long n, float *out)
{
    if (!s || (n > 0 && (!X || !out))) return fail(EU3D_ERR_ARG, "null argument");
    if (n <= 0) return EU3D_OK;
    CK(cudaSetDevice(s->dev));
    int rc;
    if ((rc = sur_ensure_io(s, n))) return rc;
    CK(cudaMemcpyAsync(s->in_d, X, (size_t)n * SUR_IN * sizeof(float), cudaMemcpyHostToDevice, s->st));
    if ((rc = eu3d_sur_infer(s, s->in_d, n, s->out_d, nullptr))) return rc;
    CK(cudaMemcpyAsync(out, s->out_d, (size_t)n * SUR_OUT * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return sur_check_err(s);
}

int eu3d_set_surrogate(eu3d_handle *h, eu3d_surrogate *s, int audit_stride)
{
    if (!h) return fail(EU3D_ERR_ARG, "null handle");
    if (audit_stride < 0) return fail(EU3D_ERR_ARG, "audit stride must be >= 0");
    CK(cudaSetDevice(h->dev));
    if (s) {
        if (s->dev != h->dev) return fail(EU3D_ERR_ARG, "surrogate on another device");
        if (s->quirks != h->quirks) return fail(EU3D_ERR_ARG, "surrogate trained under another quirk policy");
        // network outputs, active and fallback lists (list entries carry the
        // ghosted cell index in 30 bits)
        int rc = ensure_cell_list(h);
        if (rc) return rc;
    }
    h->sur = s;
    h->sur_gated = false;
    h->sur_audit_stride = audit_stride;
    if (s) h->elements = true;  // eu3d_sur_create loaded the element matrix on this device
    // recorded step graphs hold the previous surrogate's buffers and settings
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second);
    h->graphs.clear();
    return EU3D_OK;
}

int eu3d_set_surrogate_gate(eu3d_handle *h, double t_frozen, double y_max, unsigned species_mask, int audit_stride)
{
    if (!h) return fail(EU3D_ERR_ARG, "null handle");
    if (!(t_frozen >= 0.0) || !(y_max >= 0.0)) return fail(EU3D_ERR_ARG, "gate temperature and fraction must be >= 0");
    if (species_mask >> NS) return fail(EU3D_ERR_ARG, "species mask names a species past NS");
    if (audit_stride < 0) return fail(EU3D_ERR_ARG, "audit stride must be >= 0");
    h->gate_T = t_frozen;
    h->sur_gated = false;
    h->gate_y = y_max;
    h->gate_mask = species_mask;
    h->gate_audit = audit_stride;
    for (auto &g : h->graphs) cudaGraphExecDestroy(g.second);
    h->graphs.clear();
    return EU3D_OK;
}

int eu3d_react_surrogate(eu3d_handle *h)
{
    if (!h) return fail(EU3D_ERR_ARG, "null handle");
    return sur_chem_op(h, false);
}

}  // extern "C"
