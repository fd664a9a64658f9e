// Learned block-sparse preconditioner (learned.cu).
#pragma once

#include <vector>

#include "fsd_internal.h"

namespace fsd {

// Block-CSR products with the matrix tile streamed by bulk copies (bsr_tma.cu).
constexpr int kTileBlocks = 104;  // blocks (and rows) of a tile of the block-sparse products
constexpr int kBsrThreads = 128;  // threads per tile
struct BsrTmaArgs {
    const int* rowptr;
    const int* col;
    const float* val;
    const int* tile_row;  // ntiles + 1 row boundaries
    const int* ntiles;    // device count (launches cover the capacity)
    int N;
    const float* x;       // operand (mode 0: the saddle vector b)
    const float* b;       // mode 2: saddle input for the post step
    float* out;
    float* xs;            // mode 2: saddle output
    float* T;
    float* B;
    const float* B1;
    const float* B2;
    const float* pc;      // coefficients, spectral bound at kMaxPoly
    int m, k;
};
size_t bsr_tma_smem();
const void* bsr_tma_kernel(int mode);
int bsr_tma_prepare();
void bsr_tma_launch(int mode, const BsrTmaArgs& a, int grid, cudaStream_t st);
int bsr_tma_error();
int bsr_make_tiles(const std::vector<int>& rowptr, int N, std::vector<int>& tiles);
__global__ void k_compact_pruned(const unsigned* __restrict__ pn, const unsigned* __restrict__ plist,
                                 const float* __restrict__ A, const int* __restrict__ rowptr, int N, int* col,
                                 float* val);

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
    int poly_source = 0;      // coefficients in use: 1 network's interval, 2 least-squares fit, 3 caller's,
                              // 4 fixed interval
    float poly_ratio = -1.f;  // lower end of the Chebyshev interval as a fraction of lambda (-1: none)
    float user_ratio = -1.f;  // caller's fixed interval ratio (fsd_learned_set_interval; -1: none)
    float poly_loss_net = -1.f, poly_loss_fit = -1.f;  // held-out probe losses of the last build's check
    unsigned poly_builds = 0; // builds so far (the check's probe draws)
    cudaGraph_t pgraph = nullptr;
    cudaGraphExec_t pexec = nullptr;
    cudaGraphNode_t pnode_first = nullptr, pnode_last = nullptr;
    const void* pkey[10] = {};
    int pkey_k = -1;
    // block-CSR copy of A and the row tiles of A and G for the streamed products
    int* a_rowptr = nullptr;
    int* a_col = nullptr;
    float* a_val = nullptr;
    size_t a_cap = 0;
    int* g_tiles = nullptr;   // tile_cap + 1 row boundaries, then the count at [tile_cap + 1]
    int* a_tiles = nullptr;
    int tile_cap = 0;
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
void poly_interval_coefficients(double rho, double lambda, int k, float* c);
int poly_set_interval(fsd_handle* h, double rho);
int poly_prepare_products(fsd_handle* h);

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
// Interval ratio rho = a / lambda of the Chebyshev inner polynomial predicted
// for this configuration (exp of the mean over particles of the node head's
// first output, clamped to [kRatioMin, kRatioMax]).
int mpnn_poly_ratio(fsd_handle* h, const float4* pos, double* rho, float* log_rho);
int mpnn_ratio_train_step(fsd_handle* h, const float4* pos, float target_log_rho, float lr, float* loss,
                          float* pred_log_rho, float* host_grad);

}  // namespace fsd
