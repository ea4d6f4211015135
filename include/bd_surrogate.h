/* bd_surrogate.h -- C ABI of the learned surrogate.
 *
 * The reference has no learned part.  The surrogate is an MLP
 * n_in -> width x depth (GELU) -> n_out that maps a simulation setting
 * (phi, T_final, log t_w, log t, k) to F_s, MSD and g(r) features.  The
 * engine's own runs generate its training data, and it proposes the next
 * settings to simulate.  Training and inference run on hand-written tcgen05
 * BF16 GEMMs with FP32 accumulation and FP32 Adam.  All buffers named
 * "host" are host memory; every call synchronises its own stream. */
#ifndef BD_SURROGATE_H
#define BD_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bd_surrogate bd_surrogate;

/* n_in <= 64, n_out <= 128, width in {64, 128, 192, 256}, depth hidden
 * layers (1..8), batch a multiple of 256.  Weights: seeded uniform
 * initialisation, biases zero. */
int bd_surrogate_create(int n_in, int n_out, int width, int depth, int batch, unsigned long long seed,
                        bd_surrogate **out);
int bd_surrogate_destroy(bd_surrogate *s);
int bd_surrogate_get_stream(const bd_surrogate *s, void **stream);
/* Number of parameters: sum over layers of N_l K_l + N_l. */
int bd_surrogate_param_count(const bd_surrogate *s, long long *count);
/* Flat FP32 parameters: per layer W [N_l][K_l] (row = output) then b [N_l]. */
int bd_surrogate_get_params(bd_surrogate *s, float *params_host);
int bd_surrogate_set_params(bd_surrogate *s, const float *params_host);
/* Loss weight of each output (n_out values, default 1). */
int bd_surrogate_set_output_weights(bd_surrogate *s, const float *w_host);
/* Training set: x [n][n_in], y [n][n_out] (FP32, already normalised). */
int bd_surrogate_set_data(bd_surrogate *s, const float *x_host, const float *y_host, int n);
/* `steps` Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on random minibatches
 * of the training set; *last_loss = mean weighted squared error of the last
 * minibatch (may be NULL). */
int bd_surrogate_train(bd_surrogate *s, int steps, float lr, float *last_loss);
/* Gradients of the mean loss over exactly one batch of `batch` rows,
 * without an update, in the layout of bd_surrogate_get_params. */
int bd_surrogate_gradients(bd_surrogate *s, const float *x_host, const float *y_host, float *grad_host,
                           float *loss);
/* Outputs for n inputs: y [n][n_out]. */
int bd_surrogate_predict(bd_surrogate *s, const float *x_host, int n, float *y_host);
/* The surrogate's GEMM kernel on its own: C [M][N] = A [M][K] B [N][K]^T,
 * BF16 inputs as raw bits (K a multiple of 8), FP32 output. */
int bd_umma_gemm_bf16(const unsigned short *a_host, const unsigned short *b_host, int M, int N, int K,
                      float *c_host);

#ifdef __cplusplus
}
#endif
#endif /* BD_SURROGATE_H */
