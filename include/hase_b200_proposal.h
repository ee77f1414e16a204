/*
 * hase_b200_proposal.h -- the learned importance proposal of libhase_b200.so:
 * a small MLP that scores every (sample point, reflection slice, prism) pair,
 * trained on the GPU from the per-prism gain contributions that the
 * importance-sampled method logs, and used as the ray->prism proposal of
 * hase_calc_phi_ase_learned.  No counterpart in the reference (HASEonGPU's
 * importance distribution is the straight-line gain estimate of
 * hase_importance_weights); the estimator stays unbiased because every prism
 * with beta > 0 keeps a positive probability (a defensive mixture with the
 * beta V / d^2 prior) and each ray is weighted by the inverse probability of
 * the proposal actually used.
 *
 * Network: 12 inputs -> 64 -> 64 -> 64 (SiLU) -> 1 logit; BF16 weights and
 * activations on the tensor cores (tcgen05, FP32 accumulation in tensor
 * memory), FP32 biases and output layer.  Per sample point the logits of all
 * (slice, prism) pairs go through a softmax.
 *
 * Parameters (FP32 master copy, HASE_PROPOSAL_PARAMS floats, row-major):
 *   W1[12][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4[1]
 * (W[in][out]; the device rounds W1..W3 and w4 to BF16).
 *
 * Features of a pair (sample s, image point s_j of slice j, prism p with
 * centre c, volume V, excited fraction beta), R = radius of the mesh,
 * H = height of the medium:
 *   0..2  s / (R, R, H)            3..5  (c - s_j) / (R, R, H)
 *   6     ln(|c - s_j| / R)        7     beta
 *   8     estimated ln gain along c -> s_j (a coarse column-averaged gain
 *         field sampled at 8 points, reflections folded)
 *   9     ln(beta V / |c - s_j|^2) - ln(V_mean / R^2)   (0 when beta = 0)
 *   10    slice index / 4          11    ln(sigma_e / sigma_a) of the
 *                                        spectrally averaged gain
 */
#ifndef HASE_B200_PROPOSAL_H
#define HASE_B200_PROPOSAL_H

#include "hase_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HASE_PROPOSAL_FEATURES 12
#define HASE_PROPOSAL_HIDDEN 64
#define HASE_PROPOSAL_PARAMS (12 * 64 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1)

typedef struct hase_proposal hase_proposal;

/* A network on `device` with seeded uniform fan-in initialisation. */
hase_status hase_proposal_create(int device, uint32_t seed, hase_proposal** out);
hase_status hase_proposal_destroy(hase_proposal* net);
hase_status hase_proposal_get_params(hase_proposal* net, float* params);
hase_status hase_proposal_set_params(hase_proposal* net, const float* params);

/* Logits of `rows` explicit feature rows (host arrays [rows][12] -> [rows]). */
hase_status hase_proposal_forward(hase_proposal* net, uint32_t rows, const float* features, float* logits);

/* A training set: `groups` sample points, group g owning rows
 * offsets[g] .. offsets[g+1]-1 (offsets[0] = 0), each row a feature vector and
 * a non-negative target score (the logged gain contribution of that prism).
 * Loss of a group: w_g times the cross entropy between the normalised targets
 * and the softmax of the group's logits; a batch's loss is the mean over its
 * groups. */
typedef struct {
    uint32_t groups;
    const uint32_t* offsets;     /* [groups + 1] */
    const float* features;       /* [rows][HASE_PROPOSAL_FEATURES] */
    const float* targets;        /* [rows] */
    const float* groupWeights;   /* [groups] or NULL (all 1) */
} hase_proposal_batch;

typedef struct {
    uint32_t steps;              /* Adam steps */
    uint32_t groupsPerStep;      /* step s uses groups [k G', (k+1) G'), k = s mod (groups / G') */
    float learningRate;
    float beta1;                 /* Adam moments; 0 = 0.9 */
    float beta2;                 /* 0 = 0.999 */
    float epsilon;               /* 0 = 1e-8 */
} hase_proposal_train_desc;

/* Loss and gradient (HASE_PROPOSAL_PARAMS floats, master-vector order) of the
 * whole batch: tensor-core forward and backward products, FP32 reductions. */
hase_status hase_proposal_loss_grad(hase_proposal* net, const hase_proposal_batch* batch, float* loss, float* grad);

/* Trains the network in place (Adam on the FP32 master parameters, BF16
 * images repacked on the device after every step); lossHistory [steps] may be
 * NULL. */
hase_status hase_proposal_train(hase_proposal* net, const hase_proposal_batch* batch,
                                const hase_proposal_train_desc* train, float* lossHistory);

/* ---- the learned proposal in the phi-ASE solve ---- */

typedef struct {
    float mixture;               /* weight alpha of the beta V / d^2 prior in
                                    q = (1 - alpha) softmax + alpha prior; 0 = 0.1 */
    float fallbackVariance;      /* a sample whose first-pass per-ray relative variance
                                    (rays x relative error^2) under the learned proposal
                                    exceeds this restarts with the importance weights of
                                    hase_importance_weights; 0 = never */
    uint32_t fallbackSamples;    /* out: samples that restarted */
} hase_learned_desc;

/* hase_calc_phi_ase with the learned proposal in place of the importance
 * weights (same experiment / compute / result conventions).  Every ray is
 * weighted by the inverse probability of the quantised proposal it was drawn
 * from, so the estimate stays unbiased. */
hase_status hase_calc_phi_ase_learned(hase_context* ctx, hase_proposal* net, const hase_experiment_desc* experiment,
                                      const hase_compute_desc* compute, hase_learned_desc* learned,
                                      hase_result* result);

/* hase_calc_phi_ase that also sums every ray's contribution X per (sample,
 * slice, prism): contributions [samples][slices * P] (slices = 5 with
 * reflections, else 1), the training targets of the proposal.  result may be
 * NULL. */
hase_status hase_log_contributions(hase_context* ctx, const hase_experiment_desc* experiment,
                                   const hase_compute_desc* compute, float* contributions, hase_result* result);

/* The normalised ray->prism proposal hase_calc_phi_ase_learned draws its
 * first pass from for samples [firstSample, firstSample + count): the
 * mixture (1 - mixture) softmax(logits) + mixture beta V R_j / d^2 prior
 * (mixture 0 = the default 0.1), divided by its maximum, as FP32
 * weights [count][slices * P] -- the learned counterpart of
 * hase_importance_weights, for replaying a learned solve with the CPU
 * oracle. */
hase_status hase_learned_weights(hase_context* ctx, hase_proposal* net, uint32_t firstSample, uint32_t count,
                                 uint32_t useReflections, uint32_t monochromatic, float mixture, float* weights);

/* Network features of every (slice, prism) pair of samples
 * [firstSample, firstSample + count): features [count][slices * P][12]. */
hase_status hase_proposal_features(hase_context* ctx, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                                   uint32_t monochromatic, float* features);

#ifdef __cplusplus
}
#endif

#endif /* HASE_B200_PROPOSAL_H */
