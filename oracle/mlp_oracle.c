/*
 * mlp_oracle.c — CPU oracle of the schedule-selector MLP (12 -> 64 -> 64 -> 24,
 * ReLU hidden layers, linear output, masked mean-squared error).
 *
 * TEST INFRASTRUCTURE ONLY: checks the library's hand-written CUDA forward and
 * backward kernels (sptrsv_b200/csrc/mlp.cu).  Computed in double precision.
 *
 * Parameter layout (flat, 6552 floats), weights row-major [in][out]:
 *   W1[12][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24]
 * Inputs are normalised first: xn = (x - mean) / std.
 * Loss: L = sum_{b,c} M[b,c] (Y[b,c] - T[b,c])^2 / max(1, sum M).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NI 12
#define NH 64
#define NO 24

static void offsets(int* o)
{
    o[0] = 0;                 /* W1 */
    o[1] = o[0] + NI * NH;    /* b1 */
    o[2] = o[1] + NH;         /* W2 */
    o[3] = o[2] + NH * NH;    /* b2 */
    o[4] = o[3] + NH;         /* W3 */
    o[5] = o[4] + NH * NO;    /* b3 */
    o[6] = o[5] + NO;         /* total 6552 */
}

int mlp_oracle_nparams(void)
{
    int o[7];
    offsets(o);
    return o[6];
}

/* Forward pass; Y gets B x 24 outputs. */
void mlp_oracle_forward(const float* P, const float* mean, const float* stdv, const float* X, int B, double* Y)
{
    int o[7];
    offsets(o);
    double h1[NH], h2[NH], xn[NI];
    for (int b = 0; b < B; b++) {
        for (int i = 0; i < NI; i++) xn[i] = ((double)X[b * NI + i] - mean[i]) / stdv[i];
        for (int j = 0; j < NH; j++) {
            double s = P[o[1] + j];
            for (int i = 0; i < NI; i++) s += xn[i] * P[o[0] + i * NH + j];
            h1[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < NH; j++) {
            double s = P[o[3] + j];
            for (int i = 0; i < NH; i++) s += h1[i] * P[o[2] + i * NH + j];
            h2[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < NO; j++) {
            double s = P[o[5] + j];
            for (int i = 0; i < NH; i++) s += h2[i] * P[o[4] + i * NO + j];
            Y[b * NO + j] = s;
        }
    }
}

/* Loss and gradient with respect to every parameter (G: 6552 doubles). */
double mlp_oracle_gradient(const float* P, const float* mean, const float* stdv, const float* X, const float* T,
                           const float* M, int B, double* G)
{
    int o[7];
    offsets(o);
    memset(G, 0, sizeof(double) * o[6]);
    double msum = 0;
    for (int t = 0; t < B * NO; t++) msum += M[t];
    double denom = msum > 1 ? msum : 1;
    double loss = 0;
    double xn[NI], z1[NH], h1[NH], z2[NH], h2[NH], y[NO], dy[NO], dh2[NH], dh1[NH];
    for (int b = 0; b < B; b++) {
        for (int i = 0; i < NI; i++) xn[i] = ((double)X[b * NI + i] - mean[i]) / stdv[i];
        for (int j = 0; j < NH; j++) {
            double s = P[o[1] + j];
            for (int i = 0; i < NI; i++) s += xn[i] * P[o[0] + i * NH + j];
            z1[j] = s;
            h1[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < NH; j++) {
            double s = P[o[3] + j];
            for (int i = 0; i < NH; i++) s += h1[i] * P[o[2] + i * NH + j];
            z2[j] = s;
            h2[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < NO; j++) {
            double s = P[o[5] + j];
            for (int i = 0; i < NH; i++) s += h2[i] * P[o[4] + i * NO + j];
            y[j] = s;
            double d = s - T[b * NO + j];
            loss += M[b * NO + j] * d * d;
            dy[j] = 2.0 * M[b * NO + j] * d / denom;
        }
        for (int i = 0; i < NH; i++)
            for (int j = 0; j < NO; j++) G[o[4] + i * NO + j] += h2[i] * dy[j];
        for (int j = 0; j < NO; j++) G[o[5] + j] += dy[j];
        for (int i = 0; i < NH; i++) {
            double s = 0;
            for (int j = 0; j < NO; j++) s += dy[j] * P[o[4] + i * NO + j];
            dh2[i] = z2[i] > 0 ? s : 0;
        }
        for (int i = 0; i < NH; i++)
            for (int j = 0; j < NH; j++) G[o[2] + i * NH + j] += h1[i] * dh2[j];
        for (int j = 0; j < NH; j++) G[o[3] + j] += dh2[j];
        for (int i = 0; i < NH; i++) {
            double s = 0;
            for (int j = 0; j < NH; j++) s += dh2[j] * P[o[2] + i * NH + j];
            dh1[i] = z1[i] > 0 ? s : 0;
        }
        for (int i = 0; i < NI; i++)
            for (int j = 0; j < NH; j++) G[o[0] + i * NH + j] += xn[i] * dh1[j];
        for (int j = 0; j < NH; j++) G[o[1] + j] += dh1[j];
    }
    return loss / denom;
}
