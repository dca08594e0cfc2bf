// Learned preconditioner (K8): graph, work buffers and launchers shared by
// kernels_learned.cu and the C-ABI layer (capi_learned.cu).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mfs {

constexpr int kLIn = 16;       // input features per node
constexpr int kLHid = 64;      // hidden width
constexpr int kLLayers = 4;    // message-passing layers
constexpr int kLHead = 24;     // per-node head outputs: P (9), Q (9), R (6)

// Block graph of the permuted reduced matrix (the symmetric SpMV structure):
// row i holds entries [ptr[i], ptr[i+1]) sorted by column, diag[i] is the
// diagonal entry, mirror[e] the entry of the transposed position.
struct LGraph {
    int64_t nv;
    const int64_t *ptr, *src, *diag, *mirror;
    const int32_t *col, *flag;
    float *ea;                 // per entry: ||Hs_ij||_F (0 on the diagonal), written by the features kernel
};

struct LWork {
    double *dinv;              // 3 nv: diag(H)^{-1/2}
    float *eh;                 // 9 per entry: scaled blocks Hs_ij
    float *esum;               // 9 per node
    float *h[kLLayers + 1];    // node states (h[0]: nv x kLIn, others nv x kLHid)
    float *s[kLLayers];        // aggregated neighbour states
    float *pre[kLLayers];      // pre-activations
    float *q;                  // nv x kLHead
    float *G;                  // 9 per entry (lower entries used)
    float *dG;                 // 9 per entry
    float *dq;                 // nv x kLHead
    float *dod;                // nv x 6
    float *dh[2];              // nv x kLHid
    float *ds;                 // nv x kLHid
    float *part;               // per-CTA weight-gradient partials
};

struct LParamLayout {
    int w[kLLayers];           // offsets of W_l (kLHid x (2 din + 10))
    int vh;                    // kLHead x (kLHid + 1)
    int ve;                    // 9 x 10
    int vd;                    // 6 x 10
    int total;
};

LParamLayout lpc_layout();
int lpc_layer_in(int l);
int lpc_dense_parts();
int lpc_head_parts();
void lpc_features(const LGraph &g, const double *Ax, LWork &w, cudaStream_t st);
void lpc_forward(const LGraph &g, const __nv_bfloat16 *wb, LWork &w, cudaStream_t st);
void lpc_backward(const LGraph &g, const __nv_bfloat16 *wb, LWork &w, float *grad, cudaStream_t st);
// Y = G X or G^T X over 3 nv rows (ld, nrhs); pre scales X rows, post scales Y rows (nullable)
void lpc_gmv(const LGraph &g, const float *G, bool trans, const double *X, double *Y, int64_t ld, int nrhs,
             const double *pre, const double *post, cudaStream_t st);
void lpc_scale_rows(const double *in, const double *s, bool inv, double *out, int64_t n, int nrhs, int64_t ld,
                    cudaStream_t st);
void lpc_dg(const LGraph &g, const double *Z, const double *GY, const double *GZ, const double *BS, int64_t ld,
            int nrhs, float *dG, cudaStream_t st);
void lpc_adam(float *w, __nv_bfloat16 *wb, float *m, float *v, const float *grad, int n, float lr, int step,
              cudaStream_t st);
void lpc_to_bf16(const float *w, __nv_bfloat16 *wb, int n, cudaStream_t st);

}  // namespace mfs
