// eigen.cu -- FP64 eigendecomposition of a reversible rate matrix on the GPU (one CTA).
//
// Replaces ModelMarkov::decomposeRateMatrix for reversible models (model/modelmarkov.cpp:
// 1389-1630, utils/eigendecomposition.cpp:165-320): Q is built from the exchangeabilities and
// frequencies (q_ij = s_ij pi_j, zero row sums, mean rate 1), states with pi <= 1e-10 are
// split off with eigenvalue 0 and identity eigenvectors, the rest is symmetrised as
// A = diag(sqrt pi) Q diag(1/sqrt pi) and diagonalised by cyclic Jacobi rotations.  Output
// convention as in the reference: evec[i][j] = V[i][j] / sqrt(pi_i),
// inv_evec[i][j] = V[j][i] * sqrt(pi_j), Q = evec diag(eval) inv_evec.
// The basis differs from tred2/tqli by column order and sign; likelihoods do not depend on it.
#include <cmath>
#include <vector>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr double kZeroFreq = 1e-10;
constexpr int kMaxSweeps = 60;

__device__ void jacobi_one(int n, const double *exch_upper, const double *freq_in, double *out,
                           int *flag);

__global__ void k_jacobi(int n, const double *exch_upper, const double *freq_in, double *out,
                         int *flag) {
  jacobi_one(n, exch_upper, freq_in, out, flag);
}

// one candidate model per CTA: exch[i] at exch + i * n(n-1)/2, freq[i] at freq + i * n, the
// eigensystem into out[i]
struct EigJob {
  double *out;
  int *flag;
};
__global__ void k_jacobi_batch(int n, const double *exch, const double *freq,
                               const EigJob *jobs) {
  const int i = blockIdx.x, nu = n * (n - 1) / 2;
  jacobi_one(n, exch + (size_t)i * nu, freq + (size_t)i * n, jobs[i].out, jobs[i].flag);
}

__device__ void jacobi_one(int n, const double *exch_upper, const double *freq_in, double *out,
                           int *flag) {
  extern __shared__ double sm[];
  const int ld = kMaxStates + 1;
  double *A = sm;                 // [m][ld]
  double *V = A + kMaxStates * ld;  // [m][ld]
  double *pi = V + kMaxStates * ld;  // [n]
  double *sq = pi + kMaxStates;      // [m]
  __shared__ int idx[kMaxStates];
  __shared__ int m_sh;
  __shared__ double rot[4];  // c, s, p, q
  __shared__ double offn;
  const int t = threadIdx.x;
  if (t == 0) {
    double sum = 0;
    for (int i = 0; i < n; i++) sum += freq_in[i];
    int m = 0;
    for (int i = 0; i < n; i++) {
      pi[i] = freq_in[i] / sum;
      if (pi[i] > kZeroFreq) idx[m++] = i;
    }
    m_sh = m;
  }
  __syncthreads();
  const int m = m_sh;
  // rate matrix restricted to the kept states, normalised
  for (int k = t; k < m * m; k += blockDim.x) {
    const int a = k / m, b = k % m;
    const int i = idx[a], j = idx[b];
    double s = 0.0;
    if (i != j) {
      const int lo = i < j ? i : j, hi = i < j ? j : i;
      const int u = lo * n - lo * (lo + 1) / 2 + (hi - lo - 1);
      s = exch_upper[u];
    }
    A[a * ld + b] = s * pi[j];
  }
  __syncthreads();
  if (t == 0) {
    double tot = 0;
    for (int a = 0; a < m; a++) {
      double r = 0;
      for (int b = 0; b < m; b++)
        if (b != a) r += A[a * ld + b];
      A[a * ld + a] = -r;
      tot += r * pi[idx[a]];
    }
    offn = 1.0 / tot;
    for (int a = 0; a < m; a++) sq[a] = sqrt(pi[idx[a]]);
  }
  __syncthreads();
  for (int k = t; k < m * m; k += blockDim.x) {
    const int a = k / m, b = k % m;
    A[a * ld + b] *= offn;
    V[a * ld + b] = (a == b) ? 1.0 : 0.0;
  }
  __syncthreads();
  // symmetrise: A_ab = sqrt(pi_a) Q_ab / sqrt(pi_b), averaged with the transpose
  for (int k = t; k < m * m; k += blockDim.x) {
    const int a = k / m, b = k % m;
    if (a < b) {
      const double x = sq[a] * A[a * ld + b] / sq[b];
      const double y = sq[b] * A[b * ld + a] / sq[a];
      const double v = 0.5 * (x + y);
      A[a * ld + b] = v;
      A[b * ld + a] = v;
    }
  }
  __syncthreads();
  // cyclic Jacobi sweeps
  for (int sweep = 0; sweep < kMaxSweeps; sweep++) {
    if (t == 0) {
      double off = 0, dia = 0;
      for (int a = 0; a < m; a++)
        for (int b = 0; b < m; b++) {
          const double v = A[a * ld + b] * A[a * ld + b];
          if (a == b) dia += v; else off += v;
        }
      offn = (off <= 1e-30 * dia) ? -1.0 : off;
    }
    __syncthreads();
    if (offn < 0) break;
    for (int p = 0; p < m - 1; p++) {
      for (int q = p + 1; q < m; q++) {
        if (t == 0) {
          const double apq = A[p * ld + q];
          double c = 1.0, s = 0.0;
          if (apq != 0.0) {
            const double theta = (A[q * ld + q] - A[p * ld + p]) / (2.0 * apq);
            const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(tt * tt + 1.0);
            s = tt * c;
          }
          rot[0] = c;
          rot[1] = s;
        }
        __syncthreads();
        const double c = rot[0], s = rot[1];
        if (s != 0.0) {
          // A <- J^T A J : rows p,q then columns p,q
          for (int k = t; k < m; k += blockDim.x) {
            const double ap = A[p * ld + k], aq = A[q * ld + k];
            A[p * ld + k] = c * ap - s * aq;
            A[q * ld + k] = s * ap + c * aq;
          }
          __syncthreads();
          for (int k = t; k < m; k += blockDim.x) {
            const double ap = A[k * ld + p], aq = A[k * ld + q];
            A[k * ld + p] = c * ap - s * aq;
            A[k * ld + q] = s * ap + c * aq;
            const double vp = V[k * ld + p], vq = V[k * ld + q];
            V[k * ld + p] = c * vp - s * vq;
            V[k * ld + q] = s * vp + c * vq;
          }
        }
        __syncthreads();
      }
    }
  }
  if (t == 0 && offn >= 0) atomicExch(flag, 1);  // not converged (reported, still usable)
  // expand back to n states
  double *eval = out, *evec = out + n, *inv = out + n + n * n;
  for (int k = t; k < n * n; k += blockDim.x) {
    evec[k] = ((k / n) == (k % n)) ? 1.0 : 0.0;
    inv[k] = evec[k];
  }
  for (int k = t; k < n; k += blockDim.x) eval[k] = 0.0;
  __syncthreads();
  for (int k = t; k < m * m; k += blockDim.x) {
    const int a = k / m, b = k % m;
    const int i = idx[a], j = idx[b];
    evec[i * n + j] = V[a * ld + b] / sq[a];
    inv[i * n + j] = V[b * ld + a] * sq[b];
  }
  for (int a = t; a < m; a += blockDim.x) eval[idx[a]] = A[a * ld + a];
}

}  // namespace

int launch_eigen(Session *s, const double *exch_upper, const double *freq) {
  const int n = s->desc.nstates;
  const int nu = n * (n - 1) / 2;
  double *d_in = nullptr;
  GEMS_CUDA(cudaMalloc(&d_in, sizeof(double) * (nu + n)));
  cudaError_t e = cudaMemcpyAsync(d_in, exch_upper, sizeof(double) * nu, cudaMemcpyHostToDevice,
                                  s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_in + nu, freq, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream);
  const size_t smem = sizeof(double) * (2 * kMaxStates * (kMaxStates + 1) + 2 * kMaxStates);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream);
  if (e == cudaSuccess) {
    k_jacobi<<<1, 128, smem, s->stream>>>(n, d_in, d_in + nu, s->d_model, s->d_flag);
    s->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(d_in);
  if (e != cudaSuccess) return cuda_status(e, "eigen");
  return GEMS_OK;
}

// every session's eigensystem in one launch (one CTA each), on the first session's stream
int launch_eigen_batch(Session *const *ss, int nsess, const double *exch_upper,
                       const double *freq) {
  const int n = ss[0]->desc.nstates;
  const size_t nu = (size_t)n * (n - 1) / 2;
  for (int i = 0; i < nsess; i++) GEMS_CUDA(cudaStreamSynchronize(ss[i]->stream));
  cudaStream_t st = ss[0]->stream;
  const size_t in_bytes = sizeof(double) * nsess * (nu + n);
  char *d_buf = nullptr;
  GEMS_CUDA(cudaMalloc(&d_buf, in_bytes + sizeof(EigJob) * nsess));
  double *d_exch = reinterpret_cast<double *>(d_buf), *d_freq = d_exch + nsess * nu;
  EigJob *d_jobs = reinterpret_cast<EigJob *>(d_buf + in_bytes);
  std::vector<EigJob> jobs(nsess);
  for (int i = 0; i < nsess; i++) jobs[i] = {ss[i]->d_model, ss[i]->d_flag};
  const size_t smem = sizeof(double) * (2 * kMaxStates * (kMaxStates + 1) + 2 * kMaxStates);
  cudaError_t e = cudaMemcpyAsync(d_exch, exch_upper, sizeof(double) * nsess * nu,
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_freq, freq, sizeof(double) * nsess * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(EigJob) * nsess, cudaMemcpyHostToDevice, st);
  for (int i = 0; i < nsess && e == cudaSuccess; i++)
    e = cudaMemsetAsync(ss[i]->d_flag, 0, sizeof(int), st);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_jacobi_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
  if (e == cudaSuccess) {
    k_jacobi_batch<<<nsess, 128, smem, st>>>(n, d_exch, d_freq, d_jobs);
    ss[0]->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_buf);
  if (e != cudaSuccess) return cuda_status(e, "eigen batch");
  return GEMS_OK;
}

}  // namespace gems
