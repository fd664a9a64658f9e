// Learned block-sparse preconditioner (learned.cu).
#pragma once

#include "fsd_internal.h"

namespace fsd {

struct LearnedState {
    // G in block-CSR over particles (original order), 6x6 row-major fp32 blocks
    int* g_rowptr = nullptr;
    int* g_col = nullptr;
    float* g_val = nullptr;
    int g_nnzb = 0, g_cap = 0;
    bool g_user = false;  // blocks were set through fsd_precond_set_blocks
    // R_FU^pruned + D operator (owned by the IC(0) state, pruned-list order)
    const unsigned* a_pn = nullptr;
    const unsigned* a_plist = nullptr;
    const float* a_blocks = nullptr;
    // inner GMRES work space
    int inner_cap = -1;
    float* Vi = nullptr;      // (kMaxInner + 1) x 6N basis, unnormalised
    float* Zi = nullptr;      // kMaxInner x 6N, Z_j = G V_j / |V_j|
    double* part = nullptr;   // (kMaxInner + 1) x blocks partial sums
    double* H = nullptr;      // (kMaxInner + 1) x kMaxInner Hessenberg, column-major by step, beta, y
    double* nrm = nullptr;    // kMaxInner + 1 basis norms
    unsigned* ticket = nullptr;  // last-block counter, zero between kernels
    void* mp = nullptr;      // message-passing network state (mpnn.cu)
    // two-hop sparse approximate inverse (spai.cu)
    int* sp_sets = nullptr;          // N x kSpaiCap members, particle itself first
    unsigned* sp_size = nullptr;     // N set sizes
    unsigned* sp_rowptr = nullptr;   // N + 1
    unsigned* sp_scan = nullptr;
    int* sp_bucket = nullptr;        // bucket lists
    unsigned* sp_cnt = nullptr;      // bucket counts, truncated sets, failed rows
    unsigned* sp_host = nullptr;
    int sp_truncated = 0;
    // inner solve replayed as a CUDA graph; its first and last kernel nodes
    // are re-pointed at each application's vectors
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphNode_t node_rhs = nullptr, node_post = nullptr;
    const void* gkey[8] = {};
    int gkey_k = -1;
    int captures = 0;
    // learned Chebyshev polynomial inner solve (poly.cu)
    float* pc = nullptr;      // kMaxPoly coefficients, then the spectral bound lambda of AG
    float* pbuf = nullptr;    // 5 x 6N: t, G products, three Clenshaw slots
    double* ppart = nullptr;  // block partial sums of the power iteration
    double* pnrm = nullptr;
    unsigned* pticket = nullptr;
    bool poly_user = false;   // coefficients set through fsd_learned_set_poly (else the network's)
    int poly_source = 0;      // coefficients in use: 1 network, 2 least-squares fit, 3 caller's
    float poly_loss_net = -1.f, poly_loss_fit = -1.f;  // held-out probe losses of the last build's check
    unsigned poly_builds = 0; // builds so far (the check's probe draws)
    cudaGraph_t pgraph = nullptr;
    cudaGraphExec_t pexec = nullptr;
    cudaGraphNode_t pnode_first = nullptr, pnode_last = nullptr;
    const void* pkey[8] = {};
    int pkey_k = -1;
};

LearnedState* learned(fsd_handle* h);
void learned_free(fsd_handle* h);
int learned_reserve(fsd_handle* h, int nnzb);
int learned_set_blocks(fsd_handle* h, int nnzb, const int* d_rowptr, const int* d_col, const float* d_val);
int precond_apply_learned(fsd_handle* h, const float* b, float* x);
int precond_build_learned(fsd_handle* h, const float4* pos);
int learned_set_weights(fsd_handle* h, const float* host_w, int n);
bool precond_is_flexible(const fsd_handle* h);
int spai_build(fsd_handle* h);

// poly.cu
int poly_alloc(fsd_handle* h);
void poly_free(LearnedState* s);
bool poly_active(const fsd_handle* h);
int poly_lambda(fsd_handle* h);
int poly_apply(fsd_handle* h, const float* b, float* x);
int poly_set_coefficients(fsd_handle* h, const float* host_c, int k);
int poly_get_coefficients(fsd_handle* h, float* host_c, int n);

// mpnn.cu
void mpnn_free(fsd_handle* h);
int mpnn_set_weights(fsd_handle* h, const float* host_w, int n);
int mpnn_get_weights(fsd_handle* h, float* host_w, int n);
bool mpnn_loaded(fsd_handle* h);
int mpnn_get_state(fsd_handle* h, float* host, int n, int* t);
int mpnn_set_state(fsd_handle* h, const float* host, int n, int t);
void mpnn_use_umma(fsd_handle* h, bool on);
int mpnn_infer(fsd_handle* h, const float4* pos, const unsigned* a_pn, const unsigned* a_plist, const float* a_blocks);
int mpnn_train_step(fsd_handle* h, const float4* pos, const float* host_probes, int P, uint32_t step, float lr,
                    float* loss_out, float* host_grad);
// Polynomial coefficients for this configuration from the network (mean over
// particles of the node head's first k outputs) into pc[0:k].
int mpnn_poly_coeffs(fsd_handle* h, const float4* pos, float* pc, int k);
int mpnn_poly_train_step(fsd_handle* h, const float4* pos, int P, uint32_t step, float lr, int k, int natural,
                         float* loss_out, float* loss_opt_out, float* host_grad, float* host_coef,
                         float* host_coef_opt);
int mpnn_poly_calibrate(fsd_handle* h, int k, uint32_t step);

}  // namespace fsd
