/*
 * C ABI of the learned period-proposal network's device steps (libbls_b200.so).
 *
 * No counterpart in the reference: cuPeriod searches every trial period.  The
 * network restricts the full BLS grid to the log-period windows it ranks
 * highest (cuperiod_b200/proposal.py drives these steps; the exact search of
 * the windows, and of the full grid for curves the network is unsure of, runs
 * through the entry points of bls_b200.h).
 *
 * Every pointer is a device pointer unless stated; every call is asynchronous on
 * `stream` (a cudaStream_t; NULL is the legacy default stream) and returns
 * PN_OK, PN_E_INVALID (arguments) or PN_E_CUDA (a launch failed).  A GEMM whose
 * waits ran out (a fault of the pipeline, never seen in normal operation) sets
 * *error_flag to 1 and leaves its output incomplete.
 */
#ifndef BLS_PROPOSAL_H
#define BLS_PROPOSAL_H

#ifdef __cplusplus
extern "C" {
#endif

enum { PN_OK = 0, PN_E_INVALID = 1, PN_E_CUDA = 2 };

/* GEMM output modes. */
enum { PN_OUT_BF16 = 0, PN_OUT_F32 = 1, PN_OUT_F32_ADD = 2 };

/* No counterpart in the reference.  out[m, n] = epilogue(sum_k A[m, k] B[n, k])
 * on the tensor cores (bf16 operands, fp32 accumulation): A is M x K with row
 * stride lda, B is N x K with row stride ldb (bf16, elements; strides multiples
 * of 8, base addresses 16-byte aligned).  Epilogue: + bias[n] (fp32, optional),
 * ReLU (relu != 0), times (mask[m, n] > 0) for a bf16 mask with the output's
 * stride (optional), then a bf16 store (PN_OUT_BF16), an fp32 store
 * (PN_OUT_F32) or an fp32 atomic add (PN_OUT_F32_ADD: K is split `splits` ways,
 * the output must start at zero, no ReLU or mask; the bias is added once).
 * transpose_out != 0 stores element (m, n) at out[n * ldo + m]. */
int pn_gemm(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K,
            int splits, void* out, long long ldo, int out_mode, int transpose_out,
            const float* bias, int relu, const void* mask, int* error_flag, void* stream);

/* No counterpart in the reference.  Each curve (host-side packing: t and y FP64,
 * curve c at [offsets[c], offsets[c + 1])) binned into n_bins equal time bins
 * over its own span: out[c][i][0] = the bin's mean flux minus the curve's mean,
 * over its standard deviation (0 when empty), out[c][i][1] = 1 when occupied
 * (bf16).  n_bins <= 8192. */
int pn_bin_curves(const double* t, const double* y, const long long* offsets, int n_curves,
                  int n_bins, void* out, void* stream);

/* No counterpart in the reference.  Patches of the width-7, stride-2,
 * padding-3 convolution of X (B x L_in x C, bf16, L_in even):
 * A[(b * L_in/2 + o) * kp + k * C + c] = X[b][2o + k - 3][c], zero outside and in
 * columns 7C .. kp-1 (kp a multiple of 8). */
int pn_im2col(const void* X, void* A, int B, int L_in, int C, int kp, void* stream);

/* No counterpart in the reference.  The input gradient of that convolution from
 * the gradient of its patches (layout of pn_im2col), times (act > 0) where act
 * (B x L_in x C, the ReLU output that was the convolution's input) is given. */
int pn_col2im(const void* dcol, const void* act, void* dX, int B, int L_in, int C, int kp,
              void* stream);

/* No counterpart in the reference.  out[c * ld_out + r] = in[r * ld_in + c],
 * r < R, c < C (bf16). */
int pn_transpose(const void* in, long long ld_in, void* out, long long ld_out, long long R,
                 long long C, void* stream);

/* No counterpart in the reference.  db[n] += sum over m < M of g[m * ld + n]
 * (g bf16, db fp32). */
int pn_colsum(const void* g, long long ld, long long M, int N, float* db, void* stream);

/* No counterpart in the reference.  Per row of logits (fp32, rows x n_cls): the
 * cross-entropy against labels[row] with `side` of the target on each
 * neighbouring class, added to *loss; dlogits = (softmax - target) * scale
 * (bf16). */
int pn_softmax_xent(const float* logits, int rows, int n_cls, const int* labels, float side,
                    float scale, void* dlogits, float* loss, void* stream);

/* No counterpart in the reference.  One Adam step (decoupled weight decay wd,
 * bias corrections of step `step` >= 1) on n fp32 weights w with moments m, v
 * and gradient g; w16 (bf16, optional) receives the updated weights. */
int pn_adam(float* w, float* m, float* v, const float* g, void* w16, long long n, float lr,
            float b1, float b2, float eps, float wd, int step, void* stream);

/* No counterpart in the reference.  Per row of logits: the k largest classes,
 * largest first (index, rows x k), and the softmax mass they hold (mass, rows). */
int pn_topk(const float* logits, int rows, int n_cls, int k, int* index, float* mass,
            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BLS_PROPOSAL_H */
