// Exact top-K sparsification of the SPLR Hessian, built directly in CSR.
//
// Replaces (reference benben-cd/curegot_backward, src/sinkhorn_splr_kernel.cu):
//   T_fused_kernel's Tvalues/Tflatind output       :214-345
//   launch_H_sparsification (cub::DeviceTopK, thrust::sort_by_key,
//     write_diagonal_kernel)                        :554-675
//   recompute_nonzero_values_kernel                 :681-734  (refresh_all_kernel)
//   extract_columns_and_count_kernel + DeviceScan   :741-820
//
// Design: T_t values are never materialised.  The K-th largest value is found
// by a most-significant-digit radix select over the FP64 bit patterns of
// T_ij (T >= 0, so the bit pattern orders like the value), 12-bit digits,
// each level a histogram pass that recomputes T from M and the duals.  If
// whole-value ties remain, the select continues on the flat Hsl index
// (smaller index first), so the final selection is a per-element predicate
//     key > tv  ||  (key == tv && idx' >= ti),   idx' = 2^31 - 1 - flat,
// which needs no global ordering.  A count pass and two small prefix kernels
// give every (row tile, column) and (row, column tile) its output offset, and
// the emit pass writes the CSR rows (n+j: entries i ascending, then the
// diagonal) and the per-row lists (i: entries j ascending) in place — no sort.
// The reference leaves tie order unspecified (DeviceTopK with
// determinism::not_guaranteed); this selection is deterministic.
#include <algorithm>

#include "sparsify.cuh"

namespace cg {

namespace {

constexpr int kTile = 256;  // rows and columns per count/emit tile
constexpr int kBins = 4096;

struct Digit {
  int shift, width;
};
// value digits (63 bits, sign bit is 0), then index digits (31 bits)
__device__ __forceinline__ Digit digit_of(int level) {
  switch (level) {
    case 0: return {51, 12};
    case 1: return {39, 12};
    case 2: return {27, 12};
    case 3: return {15, 12};
    case 4: return {3, 12};
    case 5: return {0, 3};
    case 6: return {19, 12};
    case 7: return {7, 12};
    default: return {0, 7};
  }
}

// T_ij with its sign bit cleared.  T >= 0 for finite inputs, so this is the
// value itself; a NaN (non-finite M or duals) may carry a sign bit, and the
// radix select's value digits assume a clear one: with it cleared, the
// histogram, count and emit passes all order every key the same way and the
// selection holds exactly Ks entries.
template <typename TM>
__device__ __forceinline__ double t_at(const TM* __restrict__ M, int i, int j, int m, double as,
                                       double bs, double s2, const double* tab) {
  return fabs(exp2_f64_sel(fma(-ld1(M + (size_t)i * m + j), s2, as + bs), tab));
}

__device__ __forceinline__ unsigned int flat_prime(int n, int H, int i, int j) {
  const unsigned int flat = (unsigned int)((long long)(n + j) * H + i);
  return 0x7FFFFFFFu - flat;
}

__device__ __forceinline__ bool selected(unsigned long long key, unsigned int idxp,
                                         const SelState& s) {
  return key > s.tv || (key == s.tv && idxp >= s.ti);
}

__global__ void sel_init_kernel(SelState* s, unsigned int* hist, long long Ks, long long Te) {
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0u;
  if (threadIdx.x == 0) {
    s->prefix = 0ull;
    s->krem = Ks;
    s->level = 0;
    s->pad = 0;
    if (Ks >= Te) {  // everything
      s->done = 1;
      s->tv = 0ull;
      s->ti = 0u;
    } else if (Ks <= 0) {  // nothing
      s->done = 1;
      s->tv = ~0ull;
      s->ti = 0xFFFFFFFFu;
    } else {
      s->done = 0;
      s->tv = 0ull;
      s->ti = 0u;
    }
  }
}

template <typename TM>
__global__ void __launch_bounds__(kThreads) hist_kernel(const TM* __restrict__ M,
                                                        const double* __restrict__ gamma, int n,
                                                        int m, double s2, const SelState* sel,
                                                        unsigned int* __restrict__ hist) {
  __shared__ double tab[kExp2TableSize];
  __shared__ unsigned int sh[kBins];
  load_exp2_table(tab);
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) sh[b] = 0u;
  __syncthreads();
  if (ldcg(&sel->done)) return;
  const int level = ldcg(&sel->level);
  const unsigned long long prefix = sel->prefix;
  const unsigned long long tv = sel->tv;
  const Digit dg = digit_of(level);
  const int H = n + m - 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
  for (int i = gw; i < n; i += nw) {
    const double as = gamma[i] * s2;
    // warp-uniform trip count: every lane reaches the warp-synchronous calls
    for (int j0 = 0; j0 < m - 1; j0 += 32) {
      const int j = j0 + lane;
      int bin = -1;
      if (j < m - 1) {
        const double T = t_at(M, i, j, m, as, gamma[n + j] * s2, s2, tab);
        const unsigned long long key = (unsigned long long)__double_as_longlong(T);
        if (level < 6) {
          if ((key >> (dg.shift + dg.width)) == prefix)
            bin = (int)((key >> dg.shift) & ((1ull << dg.width) - 1));
        } else if (key == tv) {
          const unsigned int ip = flat_prime(n, H, i, j);
          if (((unsigned long long)ip >> (dg.shift + dg.width)) == prefix)
            bin = (int)((ip >> dg.shift) & ((1u << dg.width) - 1));
        }
      }
      // warp-aggregated shared-memory increment
      const unsigned int act = __ballot_sync(0xffffffffu, bin >= 0);
      if (bin >= 0) {
        const unsigned int peers = __match_any_sync(act, bin);
        if ((__ffs(peers) - 1) == lane) atomicAdd(&sh[bin], (unsigned)__popc(peers));
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kBins; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// One CTA of 1024 threads: pick the bucket holding the krem-th largest.
__global__ void __launch_bounds__(1024) select_kernel(SelState* s, unsigned int* hist) {
  __shared__ unsigned long long part[1024];
  __shared__ int sh_b;
  __shared__ unsigned long long sh_above;
  if (threadIdx.x == 0) sh_b = -1;
  if (ldcg(&s->done)) return;
  const int level = s->level;
  const Digit dg = digit_of(level);
  const int nb = 1 << dg.width;
  const int t = threadIdx.x;
  // thread t owns bins [4t, 4t + 4); suffix sums from the top
  unsigned long long c[4];
  unsigned long long mine = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = 4 * t + q;
    c[q] = (b < nb) ? hist[b] : 0ull;
    mine += c[q];
  }
  part[t] = mine;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive suffix scan
    const unsigned long long v = (t + off < 1024) ? part[t + off] : 0ull;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  const unsigned long long krem = (unsigned long long)s->krem;
  const unsigned long long after = (t + 1 < 1024) ? part[t + 1] : 0ull;  // bins above mine
  if (after < krem && part[t] >= krem) {
    unsigned long long above = after;
    for (int q = 3; q >= 0; --q) {
      if (above + c[q] >= krem) {
        sh_b = 4 * t + q;
        sh_above = above;
        break;
      }
      above += c[q];
    }
  }
  __syncthreads();
  if (t == 0 && sh_b < 0) {
    // unreachable with consistent counts; keep the current bucket and above
    s->done = 1;
    s->tv = (level < 6) ? (s->prefix << (dg.shift + dg.width)) : s->tv;
  } else if (t == 0) {
    const int b = sh_b;
    const long long kr = (long long)(krem - sh_above);
    const unsigned long long cb = hist[b];
    s->krem = kr;
    s->prefix = (s->prefix << dg.width) | (unsigned long long)b;
    if ((long long)cb == kr) {
      s->done = 1;
      if (level < 6) {
        s->tv = s->prefix << dg.shift;
        s->ti = 0u;
      } else {
        s->ti = (unsigned int)(s->prefix << dg.shift);
      }
    } else if (level == 5) {
      s->tv = s->prefix;  // full 63-bit value; continue on the index
      s->prefix = 0ull;
      s->level = 6;
    } else {
      s->level = level + 1;
    }
  }
  __syncthreads();
  for (int b = t; b < kBins; b += blockDim.x) hist[b] = 0u;
}

// Count pass: thread t owns column c0 + t of a 256 x 256 tile.
template <typename TM>
__global__ void __launch_bounds__(kThreads) count_kernel(const TM* __restrict__ M,
                                                         const double* __restrict__ gamma, int n,
                                                         int m, double s2, const SelState* sel,
                                                         int* __restrict__ colcnt,
                                                         int* __restrict__ rowcnt, int coltiles) {
  __shared__ double tab[kExp2TableSize];
  __shared__ int srow[kTile];
  load_exp2_table(tab);
  for (int r = threadIdx.x; r < kTile; r += blockDim.x) srow[r] = 0;
  __syncthreads();
  const SelState S = *sel;
  const int ct = blockIdx.x % coltiles, rt = blockIdx.x / coltiles;
  const int r0 = rt * kTile, r1 = min(n, r0 + kTile);
  const int j = ct * kTile + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int H = n + m - 1;
  const bool jin = j < m - 1;
  const double bs = jin ? gamma[n + j] * s2 : 0.0;
  int cnt = 0;
  for (int i = r0; i < r1; ++i) {
    bool sl = false;
    if (jin) {
      const double T = t_at(M, i, j, m, gamma[i] * s2, bs, s2, tab);
      sl = selected((unsigned long long)__double_as_longlong(T), flat_prime(n, H, i, j), S);
    }
    cnt += sl;
    const unsigned int bal = __ballot_sync(0xffffffffu, sl);
    if (lane == 0 && bal) atomicAdd(&srow[i - r0], __popc(bal));
  }
  if (jin) colcnt[(size_t)rt * (m - 1) + j] = cnt;
  __syncthreads();
  for (int r = threadIdx.x; r < r1 - r0; r += blockDim.x)
    rowcnt[(size_t)ct * n + r0 + r] = srow[r];
}

// Exclusive prefixes over tiles, in place, plus totals.
__global__ void prefix_cols_kernel(int* colcnt, int* coltot, int m1, int rowtiles) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m1; j += gridDim.x * blockDim.x) {
    int run = 0;
    for (int t = 0; t < rowtiles; ++t) {
      const int c = colcnt[(size_t)t * m1 + j];
      colcnt[(size_t)t * m1 + j] = run;
      run += c;
    }
    coltot[j] = run;
  }
}
__global__ void prefix_rows_kernel(int* rowcnt, int* rowtot, int n, int coltiles) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int run = 0;
    for (int t = 0; t < coltiles; ++t) {
      const int c = rowcnt[(size_t)t * n + i];
      rowcnt[(size_t)t * n + i] = run;
      run += c;
    }
    rowtot[i] = run;
  }
}

// Block-wide exclusive scan of len ints (1024 threads); returns the total.
__device__ long long block_exclusive_scan(const int* in, int len, int* out, long long* sh) {
  const int t = threadIdx.x;
  const int chunk = (len + 1023) / 1024;
  const int b0 = min(len, t * chunk), b1 = min(len, b0 + chunk);
  long long loc = 0;
  for (int q = b0; q < b1; ++q) loc += in[q];
  sh[t] = loc;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const long long v = (t >= off) ? sh[t - off] : 0;
    __syncthreads();
    sh[t] += v;
    __syncthreads();
  }
  long long run = sh[t] - loc;
  for (int q = b0; q < b1; ++q) {
    const int c = in[q];
    out[q] = (int)run;
    run += c;
  }
  const long long total = sh[1023];
  __syncthreads();
  return total;
}

// Row pointers and per-row list starts from the counts.  A selection larger
// than the buffers' capacity (not reachable when the count predicate and the
// select agree) leaves a diagonal-only pattern and flags the select state, so
// the emit pass writes nothing and every later kernel stays in bounds.
__global__ void __launch_bounds__(1024) scan_kernel(const int* coltot, const int* rowtot, int n,
                                                    int m, long long kcap, int* scratch_c,
                                                    int* scratch_r, int* rowptr, int* ipt,
                                                    long long* kout, SelState* sel) {
  __shared__ long long sh[1024];
  const int m1 = m - 1;
  const long long K = block_exclusive_scan(coltot, m1, scratch_c, sh);
  block_exclusive_scan(rowtot, n, scratch_r, sh);
  const bool over = K > kcap;
  for (int r = threadIdx.x; r <= n; r += blockDim.x) rowptr[r] = r;
  for (int j = threadIdx.x; j < m1; j += blockDim.x)
    rowptr[n + j + 1] = over ? n + j + 1 : n + scratch_c[j] + coltot[j] + j + 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) ipt[i] = over ? 0 : scratch_r[i];
  if (threadIdx.x == 0) {
    ipt[n] = over ? 0 : (int)K;
    *kout = over ? 0 : K;
    sel->pad = over ? 1 : 0;
  }
}

// Emit pass over 256 x 256 tiles: selection bits to shared memory, then the
// CSR rows (thread per column, rows ascending) and the per-row lists (warp per
// row, columns ascending).
template <typename TM>
__global__ void __launch_bounds__(kThreads) emit_kernel(
    const TM* __restrict__ M, const double* __restrict__ gamma, int n, int m, double s2,
    const SelState* sel, const int* __restrict__ coloff, const int* __restrict__ rowoff,
    int coltiles, const int* __restrict__ rowptr, const int* __restrict__ ipt, double* val,
    int* col, int* ij, double* iv) {
  __shared__ double tab[kExp2TableSize];
  __shared__ unsigned int bits[kTile][kWarps];
  load_exp2_table(tab);
  __syncthreads();
  const SelState S = *sel;
  if (S.pad) return;  // capacity overflow flagged by scan_kernel: nothing to emit
  const int ct = blockIdx.x % coltiles, rt = blockIdx.x / coltiles;
  const int r0 = rt * kTile, r1 = min(n, r0 + kTile);
  const int c0 = ct * kTile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int H = n + m - 1;
  const int m1 = m - 1;
  {
    const int j = c0 + threadIdx.x;
    const bool jin = j < m1;
    const double bs = jin ? gamma[n + j] * s2 : 0.0;
    for (int i = r0; i < r1; ++i) {
      bool sl = false;
      if (jin) {
        const double T = t_at(M, i, j, m, gamma[i] * s2, bs, s2, tab);
        sl = selected((unsigned long long)__double_as_longlong(T), flat_prime(n, H, i, j), S);
      }
      const unsigned int bal = __ballot_sync(0xffffffffu, sl);
      if (lane == 0) bits[i - r0][warp] = bal;
    }
  }
  __syncthreads();
  // CSR rows n+j: thread per column, rows ascending.
  {
    const int j = c0 + threadIdx.x;
    if (j < m1) {
      const double bs = gamma[n + j] * s2;
      int pos = rowptr[n + j] + coloff[(size_t)rt * m1 + j];
      for (int i = r0; i < r1; ++i) {
        if (bits[i - r0][warp] & (1u << lane)) {
          col[pos] = i;
          val[pos] = t_at(M, i, j, m, gamma[i] * s2, bs, s2, tab);
          ++pos;
        }
      }
    }
  }
  // per-row lists: warp per row, the 8 32-column segments in order.
  for (int i = r0 + warp; i < r1; i += kWarps) {
    int base = ipt[i] + rowoff[(size_t)ct * n + i];
    const double as = gamma[i] * s2;
#pragma unroll
    for (int q = 0; q < kWarps; ++q) {
      const unsigned int b = bits[i - r0][q];
      if (b & (1u << lane)) {
        const int j = c0 + q * 32 + lane;
        const int p = base + __popc(b & ((1u << lane) - 1u));
        ij[p] = j;
        iv[p] = t_at(M, i, j, m, as, gamma[n + j] * s2, s2, tab);
      }
      base += __popc(b);
    }
  }
}

__global__ void diag_kernel(const double* rows, const double* cols, int n, int m, double shift,
                            const int* rowptr, double* val, int* col) {
  const int H = n + m - 1;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x) {
    if (r < n) {
      col[r] = r;
      val[r] = rows[r] + shift;
    } else {
      const int p = rowptr[r + 1] - 1;
      col[p] = r;
      val[p] = cols[r - n] + shift;
    }
  }
}

// Fixed-pattern refresh (reference recompute_nonzero_values_kernel,
// sinkhorn_splr_kernel.cu:681-734) in one launch: blocks [0, gj) recompute
// the off-diagonal values of the CSR rows n + j (warp per row), blocks
// [gj, gj + gi) those of the per-row lists (warp per row i), the rest write
// the diagonal rows/cols + shift (as diag_kernel).  The roles touch disjoint
// entries.
template <typename TM>
__global__ void refresh_all_kernel(const TM* __restrict__ M, const double* __restrict__ gamma,
                                   int n, int m, double s2, const int* __restrict__ rowptr,
                                   int* __restrict__ col, double* __restrict__ val,
                                   const int* __restrict__ ipt, const int* __restrict__ ij,
                                   double* __restrict__ iv, const double* __restrict__ rows,
                                   const double* __restrict__ cols, double shift, int gj, int gi) {
  __shared__ double tab[kExp2TableSize];
  const int b = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (b < gj + gi) {
    load_exp2_table(tab);
    __syncthreads();
  }
  if (b < gj) {
    for (int j = b * kWarps + warp; j < m - 1; j += gj * kWarps) {
      const int r = n + j;
      const double bs = gamma[n + j] * s2;
      for (int q = rowptr[r] + lane; q < rowptr[r + 1] - 1; q += 32) {
        const int i = col[q];
        val[q] = t_at(M, i, j, m, gamma[i] * s2, bs, s2, tab);
      }
    }
  } else if (b < gj + gi) {
    const int bb = b - gj;
    for (int i = bb * kWarps + warp; i < n; i += gi * kWarps) {
      const double as = gamma[i] * s2;
      for (int q = ipt[i] + lane; q < ipt[i + 1]; q += 32) {
        const int j = ij[q];
        iv[q] = t_at(M, i, j, m, as, gamma[n + j] * s2, s2, tab);
      }
    }
  } else {
    const int H = n + m - 1;
    const int gd = gridDim.x - gj - gi;
    for (int r = (b - gj - gi) * blockDim.x + threadIdx.x; r < H; r += gd * blockDim.x) {
      if (r < n) {
        col[r] = r;
        val[r] = rows[r] + shift;
      } else {
        const int p = rowptr[r + 1] - 1;
        col[p] = r;
        val[p] = cols[r - n] + shift;
      }
    }
  }
}

int grid_for(long long work, int per_block, int cap) {
  long long g = (work + per_block - 1) / per_block;
  return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

}  // namespace

size_t sparsify_work_bytes(int n, int m) {
  const int rowtiles = (n + kTile - 1) / kTile, coltiles = (m + kTile - 1) / kTile;
  size_t b = 0;
  auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
  add(kBins * sizeof(unsigned int));
  add(sizeof(SelState));
  add((size_t)rowtiles * std::max(m - 1, 1) * sizeof(int));
  add((size_t)coltiles * n * sizeof(int));
  add((size_t)std::max(m, 1) * sizeof(int));
  add((size_t)n * sizeof(int));
  add(sizeof(long long));
  add((size_t)std::max(m, 1) * sizeof(int));  // scan scratch (cols)
  add((size_t)n * sizeof(int));               // scan scratch (rows)
  return b;
}

void sparsify_work_carve(void* base, int n, int m, SparsifyWork& w) {
  const int rowtiles = (n + kTile - 1) / kTile, coltiles = (m + kTile - 1) / kTile;
  char* p = static_cast<char*>(base);
  auto take = [&](size_t bytes) {
    char* q = p;
    p += (bytes + 255) & ~size_t(255);
    return q;
  };
  w.hist = reinterpret_cast<unsigned int*>(take(kBins * sizeof(unsigned int)));
  w.sel = reinterpret_cast<SelState*>(take(sizeof(SelState)));
  w.colcnt = reinterpret_cast<int*>(take((size_t)rowtiles * std::max(m - 1, 1) * sizeof(int)));
  w.rowcnt = reinterpret_cast<int*>(take((size_t)coltiles * n * sizeof(int)));
  w.coltot = reinterpret_cast<int*>(take((size_t)std::max(m, 1) * sizeof(int)));
  w.rowtot = reinterpret_cast<int*>(take((size_t)n * sizeof(int)));
  w.kout = reinterpret_cast<long long*>(take(sizeof(long long)));
  w.scr_c = reinterpret_cast<int*>(take((size_t)std::max(m, 1) * sizeof(int)));
  w.scr_r = reinterpret_cast<int*>(take((size_t)n * sizeof(int)));
}

template <typename TM>
static int select_and_build_t(const TM* M, const double* gamma, const double* rows,
                              const double* cols, int n, int m, double s2, double shift,
                              long long Ks, SpHess& h, const SparsifyWork& w, cudaStream_t st) {
  const int rowtiles = (n + kTile - 1) / kTile, coltiles = (m + kTile - 1) / kTile;
  const long long Te = (long long)n * (m - 1);
  const int sms = 148;
  int* scr_c = w.scr_c;
  int* scr_r = w.scr_r;

  { sel_init_kernel<<<1, 256, 0, st>>>(w.sel, w.hist, Ks, Te); cg::count_launch(); }
  if (Te > 0) {
    const int hgrid = grid_for(n, kWarps, sms * 8);
    for (int level = 0; level < 9; ++level) {
      { hist_kernel<TM><<<hgrid, kThreads, 0, st>>>(M, gamma, n, m, s2, w.sel, w.hist); cg::count_launch(); }
      { select_kernel<<<1, 1024, 0, st>>>(w.sel, w.hist); cg::count_launch(); }
    }
    { count_kernel<TM><<<rowtiles * coltiles, kThreads, 0, st>>>(M, gamma, n, m, s2, w.sel,
                                                               w.colcnt, w.rowcnt, coltiles); cg::count_launch(); }
    { prefix_cols_kernel<<<grid_for(m - 1, 256, sms * 4), 256, 0, st>>>(w.colcnt, w.coltot, m - 1,
                                                                       rowtiles); cg::count_launch(); }
  }
  { prefix_rows_kernel<<<grid_for(n, 256, sms * 4), 256, 0, st>>>(w.rowcnt, w.rowtot, n,
                                                                 Te > 0 ? coltiles : 0); cg::count_launch(); }
  { scan_kernel<<<1, 1024, 0, st>>>(w.coltot, w.rowtot, n, m, h.kcap, scr_c, scr_r, h.rowptr,
                                   h.ipt, w.kout, w.sel); cg::count_launch(); }
  if (Te > 0)
    { emit_kernel<TM><<<rowtiles * coltiles, kThreads, 0, st>>>(
        M, gamma, n, m, s2, w.sel, w.colcnt, w.rowcnt, coltiles, h.rowptr, h.ipt, h.val, h.col,
        h.ij, h.iv); cg::count_launch(); }
  { diag_kernel<<<grid_for(h.H, 256, sms * 4), 256, 0, st>>>(rows, cols, n, m, shift, h.rowptr,
                                                            h.val, h.col); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int sparsify_select_and_build(bool f32, const void* M, const double* gamma, const double* rows,
                              const double* cols, int n, int m, double s2, double shift,
                              long long Ks, SpHess& h, const SparsifyWork& w,
                              cudaStream_t stream) {
  if (f32)
    return select_and_build_t(static_cast<const float*>(M), gamma, rows, cols, n, m, s2, shift,
                              Ks, h, w, stream);
  return select_and_build_t(static_cast<const double*>(M), gamma, rows, cols, n, m, s2, shift,
                            Ks, h, w, stream);
}

int sparsify_refresh(bool f32, const void* M, const double* gamma, const double* rows,
                     const double* cols, int n, int m, double s2, double shift, const SpHess& h,
                     cudaStream_t st) {
  const int sms = 148;
  const int gj = (m > 1) ? grid_for(m - 1, kWarps, sms * 8) : 0;
  const int gi = (m > 1) ? grid_for(n, kWarps, sms * 8) : 0;
  const int gd = grid_for(h.H, kThreads, sms * 2);
  if (f32)
    { refresh_all_kernel<float><<<gj + gi + gd, kThreads, 0, st>>>(
        static_cast<const float*>(M), gamma, n, m, s2, h.rowptr, h.col, h.val, h.ipt, h.ij, h.iv,
        rows, cols, shift, gj, gi); cg::count_launch(); }
  else
    { refresh_all_kernel<double><<<gj + gi + gd, kThreads, 0, st>>>(
        static_cast<const double*>(M), gamma, n, m, s2, h.rowptr, h.col, h.val, h.ipt, h.ij, h.iv,
        rows, cols, shift, gj, gi); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
