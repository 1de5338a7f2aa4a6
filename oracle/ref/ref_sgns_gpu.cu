/*
 * Reference trainer kernels on the GPU (test infrastructure, never shipped).
 *
 * Compiles src/word2vec.cu unmodified and exposes a C entry point that runs
 * the reference's own skip_gram_kernel / cbow_kernel (word2vec.cu:442-646)
 * deterministically: sentence j of a batch is launched alone with a grid of
 * j + 1 blocks whose first j blocks get empty sentence ranges, so block j
 * still seeds its LCG with blockIdx.x = j exactly as in a full batch launch.
 * The oracle's sequential restatement is checked against these results.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "word2vec.cu"

volatile bool stop_sampling_flag = false;

extern "C" int ref_sgns_run_sentencewise(int cbow_mode, int dim, int win, int neg, long long vsize,
                                         float *h_syn0, float *h_syn1, const int *h_table, int64_t tsize,
                                         const float *h_exp, const int *h_sen, const int64_t *h_sent_start,
                                         int n_sent, float alpha) {
  if (tsize != table_size) return -1;
  int reduSize = 32;
  while (reduSize < dim) reduSize *= 2;
  if (reduSize != 128 || dim != 128) return -2; /* FSIZE 64 instantiation only */
  size_t rows = (size_t)vsize * dim * sizeof(float);
  float *d0 = nullptr, *d1 = nullptr, *de = nullptr;
  int *dt = nullptr, *ds = nullptr, *dl = nullptr;
  int total = (int)h_sent_start[n_sent];
  cudaMalloc(&d0, rows);
  cudaMalloc(&d1, rows);
  cudaMalloc(&de, (EXP_TABLE_SIZE + 1) * sizeof(float));
  cudaMalloc(&dt, (size_t)tsize * sizeof(int));
  cudaMalloc(&ds, (size_t)(total > 0 ? total : 1) * sizeof(int));
  cudaMalloc(&dl, (size_t)(n_sent + 1) * sizeof(int));
  cudaMemcpy(d0, h_syn0, rows, cudaMemcpyHostToDevice);
  cudaMemcpy(d1, h_syn1, rows, cudaMemcpyHostToDevice);
  cudaMemcpy(de, h_exp, 1000 * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dt, h_table, (size_t)tsize * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(ds, h_sen, (size_t)total * sizeof(int), cudaMemcpyHostToDevice);
  std::vector<int> sl(n_sent + 1);
  for (int j = 0; j < n_sent; j++) {
    for (int k = 0; k <= j; k++) sl[k] = (int)h_sent_start[j];
    sl[j + 1] = (int)h_sent_start[j + 1];
    cudaMemcpy(dl, sl.data(), (size_t)(j + 2) * sizeof(int), cudaMemcpyHostToDevice);
    if (cbow_mode)
      cbow_kernel<64><<<j + 1, dim>>>(win, dim, neg, 0, (int)tsize, (int)vsize, alpha, de, dt, nullptr,
                                      nullptr, nullptr, ds, dl, d1, d0);
    else
      skip_gram_kernel<64><<<j + 1, dim>>>(win, dim, neg, 0, (int)tsize, (int)vsize, alpha, de, dt, nullptr,
                                           nullptr, nullptr, ds, dl, d1, d0);
    if (cudaDeviceSynchronize() != cudaSuccess) return -3;
  }
  cudaMemcpy(h_syn0, d0, rows, cudaMemcpyDeviceToHost);
  cudaMemcpy(h_syn1, d1, rows, cudaMemcpyDeviceToHost);
  cudaFree(d0);
  cudaFree(d1);
  cudaFree(de);
  cudaFree(dt);
  cudaFree(ds);
  cudaFree(dl);
  return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

/* The reference's convergence similarity kernel, batch_similarity_direct_index_optimized_kernel
 * (word2vec.cu:1448-1506), launched as batch_node_neighbor_direct_index launches it
 * (word2vec.cu:1833-1842: one block per pair, 128 threads, 256 beyond 200 dims) on
 * given (node, neighbour) vertex pairs of a syn0 table in vocabulary order.
 * out[i]: the cosine of pair i.  Returns 0, or a negative CUDA failure. */
extern "C" int ref_pair_similarity(const float *h_syn0, long long vsize, int dim, const uint32_t *h_node,
                                   const uint32_t *h_nbr, int n, const uint32_t *h_id2offset, long long V,
                                   float *h_out) {
  float *d0 = nullptr, *dr = nullptr;
  vertex_id_t *dn = nullptr, *dm = nullptr, *di = nullptr;
  size_t rows = (size_t)vsize * dim * sizeof(float);
  if (cudaMalloc(&d0, rows) != cudaSuccess) return -1;
  cudaMalloc(&dr, sizeof(float) * (size_t)(n > 0 ? n : 1));
  cudaMalloc(&dn, sizeof(vertex_id_t) * (size_t)(n > 0 ? n : 1));
  cudaMalloc(&dm, sizeof(vertex_id_t) * (size_t)(n > 0 ? n : 1));
  cudaMalloc(&di, sizeof(vertex_id_t) * (size_t)V);
  cudaMemcpy(d0, h_syn0, rows, cudaMemcpyHostToDevice);
  cudaMemcpy(dn, h_node, sizeof(vertex_id_t) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dm, h_nbr, sizeof(vertex_id_t) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(di, h_id2offset, sizeof(vertex_id_t) * V, cudaMemcpyHostToDevice);
  int threads = dim > 200 ? 256 : 128;
  if (n > 0)
    batch_similarity_direct_index_optimized_kernel<<<n, threads, 3 * threads * sizeof(float)>>>(d0, dn, dm, dr, dim,
                                                                                               n, di);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess && n > 0) e = cudaMemcpy(h_out, dr, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(d0);
  cudaFree(dr);
  cudaFree(dn);
  cudaFree(dm);
  cudaFree(di);
  return e == cudaSuccess ? 0 : -2;
}
