/*
 * dsmc_surrogate.h - C ABI of the warm-start surrogate's kernels (part of
 * libdsmc_b200.so).
 *
 * No counterpart in the reference: it always starts a run from a Maxwellian
 * at rest, uniform in the empty voxels (System::setup_molecules,
 * code/base_code/program/dsmc/system.cpp:398-430).  These kernels train and
 * run a 3-level 3D U-Net that predicts the steady per-voxel density and drift
 * from the solid mask, so dsmc_particles_init_field (dsmc_b200.h) can seed
 * the particles from a local drifting Maxwellian instead.
 *
 * Conventions: every pointer is DEVICE memory of the current CUDA device;
 * `stream` is a cudaStream_t (NULL: the legacy default stream); calls are
 * enqueued and return without synchronising.  Volumes are channels-last
 * bf16 (uint16_t bit patterns) [batch][S][S][S][channels] with S a power of
 * two >= 4 (convolutions: batch*S^3 a multiple of 128), addressed by a channel stride `*_cs` and offset `*_coff` (both
 * multiples of 8, tensors 16-byte aligned), so a channel concatenation is two
 * views of one buffer.  3x3x3 convolutions pad periodically.  Weights of a
 * 3x3x3 layer are [cout][27][cin], tap t = 9*(d0+1) + 3*(d1+1) + (d2+1) for
 * the offsets d in {-1,0,1} along the slowest to fastest spatial axis.
 * Status: DSMC_OK or a DSMC_ERR_* code (message in dsmc_last_error(NULL)).
 */
#ifndef DSMC_SURROGATE_H
#define DSMC_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out[v][coff + co] = act(bias[co] + sum_{t,ci} w[co][t][ci] in[v + off(t)][ci]),
 * act = ReLU when relu != 0; then times (mask[v][mask_coff + co] > 0) when
 * mask is not NULL (the ReLU mask of a gradient).  cin in {16, 32, 48, 64, 96}
 * (a multiple of 16), cout in {16, 32, 48, 64, 96}.  bias may be NULL.
 * tcgen05.mma implicit GEMM, fp32 accumulation in tensor memory.  The
 * gradient with respect to the input is this call on the weights that
 * dsmc_sg_pack_weights writes as w_dgrad, with in = the output gradient. */
int dsmc_sg_conv3(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int cin,
                  const uint16_t *w, const float *bias, int cout, uint16_t *out, int out_cs, int out_coff, int relu,
                  const uint16_t *mask, int mask_cs, int mask_coff);

/* dw[co][t][ci] += sum_v dy[v][co] x[v + off(t)][ci] (fp32, accumulated: zero
 * dw first).  cout a multiple of 16, cin in {16, 32, 48, 64, 96}. */
int dsmc_sg_conv3_wgrad(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, int cout,
                        const uint16_t *x, int x_cs, int x_coff, int cin, float *dw);

/* db[c] += sum_v dy[v][c], c <= 128 channels. */
int dsmc_sg_bias_grad(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, int c,
                      float *db);

/* 2x2x2 average pooling of an S^3 volume into (S/2)^3, and its backward fused
 * with the skip-connection gradient and the ReLU mask of the pooled
 * activation: out[child] = (skip[child] + dy[parent] / 8) * (act[child] > 0)
 * (skip may be NULL).  S is the edge of the input (pool2) and of the output
 * (pool2_bwd). */
int dsmc_sg_pool2(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int c, uint16_t *out,
                  int out_cs, int out_coff);
int dsmc_sg_pool2_bwd(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff,
                      const uint16_t *skip, int skip_cs, int skip_coff, const uint16_t *act, int act_cs, int act_coff,
                      int c, uint16_t *out, int out_cs, int out_coff);

/* Nearest 2x upsampling of an (S/2)^3 volume into S^3 (S = output edge), and
 * its backward: out[parent] = sum of dy over the 8 children, times
 * (act[parent] > 0) when act is not NULL. */
int dsmc_sg_up2(void *stream, int batch, int S, const uint16_t *in, int in_cs, int in_coff, int c, uint16_t *out,
                int out_cs, int out_coff);
int dsmc_sg_up2_bwd(void *stream, int batch, int S, const uint16_t *dy, int dy_cs, int dy_coff, const uint16_t *act,
                    int act_cs, int act_coff, int c, uint16_t *out, int out_cs, int out_coff);

/* Network input, 16 channels: 1 in an empty voxel (solid[v] == 0), the
 * sample's scalar feature (feature[b]), zeros. */
int dsmc_sg_pack_input(void *stream, int batch, int S, const uint8_t *solid, const float *feature, uint16_t *out);

/* Output head, a 1x1x1 convolution 16 -> 4 in fp32:
 * out[v][c] = bh[c] + sum_k wh[c][k] e[v][k]. */
int dsmc_sg_head(void *stream, int batch, int S, const uint16_t *e, int e_cs, int e_coff, const float *wh,
                 const float *bh, float *out);

/* Weighted squared error over the rows with valid[v] != 0 and its backward
 * through the head: *loss += sum_v sum_c cw[c] (out - target)^2 * inv_count;
 * dwh, dbh accumulate; de[v][k] = (sum_c wh[c][k] dout[v][c]) * (e[v][k] > 0).
 * sample_coef (NULL: none): per-sample values added to dout[v][coef_channel]
 * of every valid row of the sample (dsmc_sg_sample_flux_loss's coef). */
int dsmc_sg_loss_head_bwd(void *stream, int batch, int S, const float *out, const float *target,
                          const uint8_t *valid, const float *channel_weight, float inv_count, const uint16_t *e,
                          int e_cs, int e_coff, const float *wh, float *dwh, float *dbh, uint16_t *de, int de_cs,
                          int de_coff, double *loss, const double *sample_coef, int coef_channel);

/* Per-sample mean term of the loss: with m_b the mean over sample b's valid
 * rows of out[v][channel] - target[v][channel] (the error of the sample's
 * mean drift, i.e. of its flux), *loss += weight * sum_b m_b^2 / batch and
 * coef[b] = its derivative with respect to each of those outputs, for
 * dsmc_sg_loss_head_bwd.  work: 2*batch doubles of scratch (device). */
int dsmc_sg_sample_flux_loss(void *stream, int batch, int S, const float *out, const float *target,
                             const uint8_t *valid, int channel, float weight, double *work, double *coef,
                             double *loss);

/* Adam (Kingma & Ba 2015) with bias correction, step >= 1, on n fp32 values. */
int dsmc_sg_adam(void *stream, float *param, const float *grad, float *m, float *v, int64_t n, float lr, float beta1,
                 float beta2, float eps, int64_t step);

/* fp32 master weights [cout][27][cin] -> bf16 forward weights (same layout)
 * and, when w_dgrad is not NULL, the input-gradient weights
 * w_dgrad[ci][t][co] = w[co][26 - t][ci]. */
int dsmc_sg_pack_weights(void *stream, const float *w, int cout, int cin, uint16_t *w_fwd, uint16_t *w_dgrad);

/* Error flags of the surrogate kernels (bit 0: a convolution's bounded wait
 * on its tensor-core completion ran out; bit 1: the same in the weight
 * gradient); clear != 0 resets them.  Synchronises with the device. */
int dsmc_sg_status(unsigned *error_flags, int clear);

#ifdef __cplusplus
}
#endif
#endif /* DSMC_SURROGATE_H */
