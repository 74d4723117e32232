// structure.cu -- symbolic structure of one pass (rebuilt after
// RobustDelete): the camera-grouped observation order (the reference's nro
// indexing, rbacore.cpp:401-430), the covisible camera pairs that make up
// the off-diagonal blocks of the reduced camera system (rbacore.cpp:
// 1362-1390 grow the same set into a skyline), their per-point
// contributions sorted by block, and the block rows used by the SpMV.
// Setup only: sorts and scans come from CUB.
#include <cub/cub.cuh>

#include "internal.h"

namespace rpba {

namespace {

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

int key_bits(long long maxkey) {
  int b = 1;
  while (b < 32 && (1ll << b) <= maxkey) ++b;
  return b;
}

__global__ void k_iota_key(const int *o_cam, int n, unsigned *key, int *iota) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = (unsigned)o_cam[i];
  iota[i] = i;
}

__global__ void k_hist(const int *v, int n, int *cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(cnt + v[i], 1);
}

__global__ void k_pair_count(DevLSA L, int *pcnt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > L.npts) return;
  if (p == L.npts) {
    pcnt[p] = 0;
    return;
  }
  const int t0 = L.pt_off[p], t1 = L.pt_off[p + 1];
  int c = 0;
  for (int s = t0; s < t1; ++s) {
    const int ks = L.o_cam[s];
    if (ks < L.begini) continue;
    for (int t = s + 1; t < t1; ++t) {
      const int kt = L.o_cam[t];
      if (kt >= L.begini && kt != ks) ++c;
    }
  }
  pcnt[p] = c;
}

__global__ void k_pair_emit(DevLSA L, const int *poff, unsigned *key, unsigned long long *val) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= L.npts) return;
  const int t0 = L.pt_off[p], t1 = L.pt_off[p + 1];
  int w = poff[p];
  const unsigned n = (unsigned)L.nimg;
  for (int s = t0; s < t1; ++s) {
    const int ks = L.o_cam[s];
    if (ks < L.begini) continue;
    for (int t = s + 1; t < t1; ++t) {
      const int kt = L.o_cam[t];
      if (kt < L.begini || kt == ks) continue;
      const bool sf = ks < kt;
      const unsigned kmin = sf ? ks : kt, kmax = sf ? kt : ks;
      const unsigned omin = sf ? s : t, omax = sf ? t : s;
      key[w] = kmin * n + kmax;
      val[w] = ((unsigned long long)omin << 32) | omax;
      ++w;
    }
  }
}

__global__ void k_unpack_contrib(const unsigned long long *val, long long n, int2 *contrib) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long v = val[i];
  contrib[i] = make_int2((int)(v >> 32), (int)(v & 0xffffffffu));
}

__global__ void k_block_count(const unsigned *bkey, int nb, int nimg, int *cntN, int *cntT, unsigned *tkey,
                              int *tidx) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const unsigned row = bkey[b] / (unsigned)nimg, col = bkey[b] % (unsigned)nimg;
  atomicAdd(cntN + row, 1);
  atomicAdd(cntT + col, 1);
  tkey[b] = col * (unsigned)nimg + row;
  tidx[b] = b;
}

__global__ void k_row_sizes(const int *cntN, const int *cntT, int nimg, int *rs) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nimg) return;
  rs[k] = k < nimg ? cntN[k] + cntT[k] + 1 : 0;
}

__global__ void k_fill_normal(const unsigned *bkey, int nb, int nimg, const int *rowoff, const int *cntT,
                              const int *firstN, int2 *ent) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int row = (int)(bkey[b] / (unsigned)nimg), col = (int)(bkey[b] % (unsigned)nimg);
  const int pos = rowoff[row] + cntT[row] + 1 + (b - firstN[row]);
  ent[pos] = make_int2(col, nimg + b);
}

__global__ void k_fill_transposed(const unsigned *bkey, const int *tidx_sorted, int nb, int nimg,
                                  const int *rowoff, const int *firstT, int2 *ent) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  const int b = tidx_sorted[q];
  const int row = (int)(bkey[b] / (unsigned)nimg), col = (int)(bkey[b] % (unsigned)nimg);
  const int pos = rowoff[col] + (q - firstT[col]);
  ent[pos] = make_int2(row, (int)((unsigned)(nimg + b) | 0x80000000u));
}

// Work items of the SpMV: each row's entry list cut into runs of <= 3 (the
// symmetric form: from the row's diagonal entry on, the transposed entries
// before it are served by their blocks' rows).  rowspan: (diagonal entry,
// end entry) of every row.
__global__ void k_row_items(const int *rowoff, const int *cntT, int nimg, int begini, int sym, int *cnt,
                            int2 *rowspan) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nimg) return;
  const int first = k < nimg ? rowoff[k] + (sym ? cntT[k] : 0) : 0;
  cnt[k] = (k < nimg && k >= begini) ? (rowoff[k + 1] - first + 2) / 3 : 0;
  if (k < nimg) rowspan[k] = make_int2(rowoff[k] + cntT[k], rowoff[k + 1]);
}

__global__ void k_fill_items(const int *rowoff, const int *cntT, const int *row_item_off, int nimg, int begini,
                             int sym, int4 *meta) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nimg || k < begini) return;
  const int end = rowoff[k + 1], first = rowoff[k] + (sym ? cntT[k] : 0);
  for (int t = row_item_off[k], j = 0; t < row_item_off[k + 1]; ++t, ++j) {
    const int e0 = first + 3 * j;
    meta[t] = make_int4(k, e0, min(e0 + 3, end), 0);
  }
}

// (row, column, transposed slot) of every block of the reduced camera
// system in storage order: the diagonal blocks, then the off-diagonal blocks
// (key row * n + col); the slot of an off-diagonal block is its position in
// column order (the sorted transposed keys), -1 for a diagonal block
__global__ void k_fill_bidx(const unsigned *bkey, int nb, int nimg, int4 *bidx) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nimg + nb) return;
  if (i < nimg) {
    bidx[i] = make_int4((int)i, (int)i, -1, 0);
  } else {
    const unsigned key = bkey[i - nimg];
    bidx[i] = make_int4((int)(key / (unsigned)nimg), (int)(key % (unsigned)nimg), 0, 0);
  }
}
__global__ void k_fill_slots(const int *tidx_sorted, int nb, int nimg, int4 *bidx) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  bidx[nimg + tidx_sorted[q]].z = q;
}

__global__ void k_fill_diag(int nimg, const int *rowoff, const int *cntT, int2 *ent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nimg) return;
  ent[rowoff[k] + cntT[k]] = make_int2(k, k);
}

}  // namespace

size_t structure_cub_bytes(int nobs, long long npairs, int nimg) {
  size_t m = 0, b = 0;
  const int np = (int)(npairs > 0 ? npairs : 1);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (unsigned *)nullptr, (unsigned *)nullptr, (int *)nullptr,
                                  (int *)nullptr, nobs > 0 ? nobs : 1);
  m = std::max(m, b);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (unsigned *)nullptr, (unsigned *)nullptr,
                                  (unsigned long long *)nullptr, (unsigned long long *)nullptr, np);
  m = std::max(m, b);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (unsigned *)nullptr, (unsigned *)nullptr, (int *)nullptr,
                                  (int *)nullptr, np);
  m = std::max(m, b);
  cub::DeviceRunLengthEncode::Encode(nullptr, b, (unsigned *)nullptr, (unsigned *)nullptr, (int *)nullptr,
                                     (int *)nullptr, np);
  m = std::max(m, b);
  const int ns = std::max(std::max(nimg + 1, np + 1), nobs + 1);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (int *)nullptr, (int *)nullptr, ns);
  m = std::max(m, b);
  return m + 256;
}

void build_camera_order(DevLSA &L, StructWork &S, cudaStream_t s) {
  if (L.nobs > 0) {
    k_iota_key<<<nblk(L.nobs, 256), 256, 0, s>>>(L.o_cam, L.nobs, S.ckey, S.iota);
    size_t bytes = S.cub_bytes;
    RPBA_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(S.cub_tmp, bytes, S.ckey, S.ckey2, S.iota, L.camlist, L.nobs,
                                                    0, key_bits(L.nimg), s));
  }
  RPBA_CUDA_CHECK(cudaMemsetAsync(S.ccnt, 0, sizeof(int) * (L.nimg + 1), s));
  if (L.nobs > 0) k_hist<<<nblk(L.nobs, 256), 256, 0, s>>>(L.o_cam, L.nobs, S.ccnt);
  size_t bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.ccnt, L.coff, L.nimg + 1, s));
}

int build_pairs(DevLSA &L, StructWork &S, long long max_pairs, long long *npairs_out, cudaStream_t s) {
  k_pair_count<<<nblk(L.npts + 1, 256), 256, 0, s>>>(L, S.pcnt);
  size_t bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.pcnt, S.poff, L.npts + 1, s));
  int total = 0;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&total, S.poff + L.npts, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  if (total < 0 || total > max_pairs) throw CudaError(cudaErrorInvalidValue, "pair count exceeds capacity");
  *npairs_out = total;
  if (total == 0) {
    L.nboff = 0;
    return 0;
  }
  k_pair_emit<<<nblk(L.npts, 256), 256, 0, s>>>(L, S.poff, S.pkey, S.pval);
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(S.cub_tmp, bytes, S.pkey, S.pkey2, S.pval, S.pval2, total, 0,
                                                  key_bits((long long)L.nimg * L.nimg), s));
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceRunLengthEncode::Encode(S.cub_tmp, bytes, S.pkey2, S.bkey, S.bcnt, S.nrun, total, s));
  int nb = 0;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&nb, S.nrun, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(S.bcnt + nb, 0, sizeof(int), s));
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.bcnt, S.boff, nb + 1, s));
  k_unpack_contrib<<<nblk(total, 256), 256, 0, s>>>(S.pval2, total, S.contrib);
  L.nboff = nb;
  L.boff = S.boff;
  L.contrib = S.contrib;
  return nb;
}

void build_bsr(DevLSA &L, StructWork &S, cudaStream_t s) {
  const int n = L.nimg, nb = L.nboff;
  RPBA_CUDA_CHECK(cudaMemsetAsync(S.cntN, 0, sizeof(int) * (n + 1), s));
  RPBA_CUDA_CHECK(cudaMemsetAsync(S.cntT, 0, sizeof(int) * (n + 1), s));
  if (nb > 0) k_block_count<<<nblk(nb, 256), 256, 0, s>>>(S.bkey, nb, n, S.cntN, S.cntT, S.tkey, S.tidx);
  size_t bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.cntN, S.firstN, n + 1, s));
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.cntT, S.firstT, n + 1, s));
  k_row_sizes<<<nblk(n + 1, 256), 256, 0, s>>>(S.cntN, S.cntT, n, S.rowtmp);
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.rowtmp, S.rowoff, n + 1, s));
  if (nb > 0) {
    bytes = S.cub_bytes;
    RPBA_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(S.cub_tmp, bytes, S.tkey, S.tkey2, S.tidx, S.tidx2, nb, 0,
                                                    key_bits((long long)n * n), s));
    k_fill_normal<<<nblk(nb, 256), 256, 0, s>>>(S.bkey, nb, n, S.rowoff, S.cntT, S.firstN, S.ent);
    k_fill_transposed<<<nblk(nb, 256), 256, 0, s>>>(S.bkey, S.tidx2, nb, n, S.rowoff, S.firstT, S.ent);
  }
  k_fill_diag<<<nblk(n, 256), 256, 0, s>>>(n, S.rowoff, S.cntT, S.ent);
  const int sym = L.blocks32 ? 1 : 0;
  k_row_items<<<nblk(n + 1, 256), 256, 0, s>>>(S.rowoff, S.cntT, n, L.begini, sym, S.row_items, S.rowspan);
  bytes = S.cub_bytes;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(S.cub_tmp, bytes, S.row_items, S.row_item_off, n + 1, s));
  int nitems = 0;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&nitems, S.row_item_off + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  k_fill_items<<<nblk(n, 256), 256, 0, s>>>(S.rowoff, S.cntT, S.row_item_off, n, L.begini, sym, S.item_meta);
  if (L.blocks32) {
    k_fill_bidx<<<nblk((long long)n + nb, 256), 256, 0, s>>>(S.bkey, nb, n, S.bidx);
    if (nb > 0) k_fill_slots<<<nblk(nb, 256), 256, 0, s>>>(S.tidx2, nb, n, S.bidx);
    L.bidx = S.bidx;
    L.firstN = S.firstN;
    L.firstT = S.firstT;
  }
  L.rowoff = S.rowoff;
  L.ent = S.ent;
  L.nitems = nitems;
  L.row_item_off = S.row_item_off;
  L.item_meta = S.item_meta;
  L.rowspan = S.rowspan;
}

// ---- PointXXvIn (rbacore.cpp:1918-1974) on the device: the track-ordered
// observation arrays (point major, observations in track order) of the
// points with at least two observations (in GCP mode also those with one
// and a GCP index above 0) and |Z| > 1e-8.
namespace {

__global__ void k_track_count(TrackIn T, int *cnt, int *pval, long long *pairs, int *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > T.np) return;
  if (p == T.np) {  // exclusive-scan sentinels
    cnt[p] = 0;
    pval[p] = 0;
    return;
  }
  const int s0 = T.pt_off[p], s1 = T.pt_off[p + 1];
  int c = 0;
  for (int j = s0; j < s1; ++j) {
    const int im = T.pt_img[j];
    if (im < 0 || im >= T.n) {
      atomicOr(err, 1);
      continue;
    }
    const int sl = T.pt_slot[j];
    if (sl < 0 || sl >= T.img_off[im + 1] - T.img_off[im]) atomicOr(err, 1);
    for (int jj = s0; jj < j; ++jj)
      if (T.pt_img[jj] == im) atomicOr(err, 2);  // an image twice in one track
    ++c;
  }
  const bool valid = fabs((double)T.XX[3 * p + 2]) > 1.e-8 && (c >= 2 || (T.gcp && T.gcp[p] > 0 && c > 0));
  cnt[p] = valid ? c : 0;
  pval[p] = valid ? 1 : 0;
  pairs[p] = valid ? (long long)c * (c - 1) / 2 : 0;
}

__global__ void k_track_scatter(TrackIn T, const int *ooff, const int *pidx, const int *pval, TrackOut O) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= T.np || !pval[p]) return;
  const int q = pidx[p];
  int o = ooff[p];
  O.pt_id[q] = p;
  O.pt_off[q] = o;
  if (O.gcp) O.gcp[q] = T.gcp[p];
  for (int j = 0; j < 3; ++j) O.X[3 * (size_t)q + j] = (double)T.XX[3 * (size_t)p + j];
  for (int j = T.pt_off[p]; j < T.pt_off[p + 1]; ++j, ++o) {
    const int im = T.pt_img[j], slot = T.pt_slot[j];
    const size_t sl = (size_t)T.img_off[im] + slot;
    O.o_cam[o] = im;
    O.o_slot[o] = slot;
    O.o_pt[o] = q;
    O.o_xg[o] = make_float2(T.xg[2 * sl], T.xg[2 * sl + 1]);
    O.o_w[o] = make_float4(T.wx[sl], T.wy[sl], T.wxy[sl], 0.f);
  }
}

}  // namespace

int track_count(const TrackIn &T, TrackScan &W, int *nobs, int *npts, long long *max_pairs, cudaStream_t s) {
  const int n1 = T.np + 1;
  RPBA_CUDA_CHECK(cudaMemsetAsync(W.err, 0, sizeof(int), s));
  k_track_count<<<(n1 + 255) / 256, 256, 0, s>>>(T, W.cnt, W.pval, W.pairs, W.err);
  size_t b1 = 0, b2 = 0, b3 = 0;
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, b1, W.cnt, W.ooff, n1, s));
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, b2, W.pval, W.pidx, n1, s));
  RPBA_CUDA_CHECK(cub::DeviceReduce::Sum(nullptr, b3, W.pairs, W.psum, std::max(T.np, 1), s));
  const size_t need = std::max(b1, std::max(b2, b3));
  void *tmp = nullptr;
  RPBA_CUDA_CHECK(cudaMallocAsync(&tmp, need, s));
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp, b1, W.cnt, W.ooff, n1, s));
  RPBA_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp, b2, W.pval, W.pidx, n1, s));
  RPBA_CUDA_CHECK(cub::DeviceReduce::Sum(tmp, b3, W.pairs, W.psum, std::max(T.np, 1), s));
  RPBA_CUDA_CHECK(cudaFreeAsync(tmp, s));
  int hv[3] = {0, 0, 0};
  long long hp = 0;
  RPBA_CUDA_CHECK(cudaMemcpyAsync(hv, W.ooff + T.np, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(hv + 1, W.pidx + T.np, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(hv + 2, W.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaMemcpyAsync(&hp, W.psum, sizeof(long long), cudaMemcpyDeviceToHost, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
  *nobs = hv[0];
  *npts = hv[1];
  *max_pairs = T.np > 0 ? hp : 0;
  return hv[2];
}

void track_scatter(const TrackIn &T, const TrackScan &W, const TrackOut &O, int nobs, int npts, cudaStream_t s) {
  if (T.np > 0) k_track_scatter<<<(T.np + 255) / 256, 256, 0, s>>>(T, W.ooff, W.pidx, W.pval, O);
  RPBA_CUDA_CHECK(cudaMemcpyAsync(O.pt_off + npts, &nobs, sizeof(int), cudaMemcpyHostToDevice, s));
  RPBA_CUDA_CHECK(cudaStreamSynchronize(s));
}

cudaError_t cub_exclusive_sum_int(void *tmp, size_t &bytes, const int *in, int *out, int n, cudaStream_t s) {
  return cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, s);
}

}  // namespace rpba
