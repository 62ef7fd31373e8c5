// fft_plane.cuh -- 3D real transforms by x-planes: one thread block holds a
// whole plane of the grid in shared memory.
//
//   k_plane_fwd  bulk-copies the real plane x = const (s^2 values, contiguous)
//                into shared memory with one TMA transfer, applies the
//                prologue, runs the R2C transforms along z and the C2C
//                transforms along y in shared memory, and writes the half
//                spectrum plane [y][kz] back with one TMA transfer;
//   k_plane_inv  the reverse for one or more spectrum planes (inverse y,
//                C2R along z) with the epilogues of k_z_c2r.
// Between them the x pass (k_x_roundtrip) works on the same [x][y][kz]
// layout, so a transform costs three passes over the field instead of five.
// Included by fft.cu inside namespace mpdpft (needs ZArgs, z_output and the
// Stockham helpers).
#pragma once

constexpr int kPlaneThreads = 512;
constexpr long kTmaSpinLimit = 1L << 24;  // bounded mbarrier wait (~seconds with backoff)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One 1D bulk copy global -> shared, completing on bar (issued by one thread
// after it armed bar with the byte count).
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of bar.  On timeout the error word is
// raised and the wait is retried once more (a copy may still be landing in
// this block's shared memory); false means the data must not be used.
__device__ inline bool mbar_wait(unsigned long long* bar, unsigned parity, int* err) {
  for (int round = 0; round < 2; ++round) {
    for (long i = 0; i < kTmaSpinLimit; ++i) {
      if (mbar_try_wait(bar, parity)) return round == 0;
      if (i > 32) __nanosleep(64);
    }
    if (round == 0 && err && threadIdx.x == 0) atomicExch(err, 1);
  }
  return false;
}

// Shared -> global bulk copy of `bytes` (one thread), waited for before the
// block may reuse or release the source.
__device__ __forceinline__ void tma_store_1d(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Orders this thread's generic shared-memory accesses before later
// async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tile widths (lines per fft_lines call) and the instantiated sizes: the z
// transforms (length s/2) take NLZ rows at a time, the y transforms NLY
// columns.  The columns kz = 0 and kz = s/2 are transformed together as one
// complex column (both are real before the forward y transform and after the
// inverse one), so the y pass runs exactly s/2 columns.
template <typename R>
constexpr int plane_nly(int s) { return (sizeof(R) == sizeof(float) && s >= 128) ? 32 : 16; }
template <typename R>
constexpr int plane_nlz(int s) { return 2 * plane_nly<R>(s); }

template <typename R>
inline bool plane_size_instantiated(int s) {
  return s == 32 || s == 64 || (sizeof(R) == sizeof(float) && s == 128);
}

// Shared-memory bytes: the spectrum plane (which first holds the real plane),
// the two Stockham tiles, twiddles, and the |grad|^2 accumulator (inverse,
// EPI_GRAD) or the epilogue tile (inverse, Coulomb epilogues).
template <typename R>
__host__ __device__ constexpr size_t plane_tile(int S, int NLY, int NLZ) {
  return (size_t)S * (NLY + 1) > (size_t)(S / 2) * (NLZ + 1) ? (size_t)S * (NLY + 1) : (size_t)(S / 2) * (NLZ + 1);
}
template <typename R>
__host__ __device__ constexpr size_t plane_fwd_smem(int S, int NLY, int NLZ) {
  return ((size_t)S * (S / 2 + 1) + 2 * plane_tile<R>(S, NLY, NLZ) + 2 * (size_t)S + (size_t)(S / 2)) * 2 * sizeof(R);
}
template <typename R>
__host__ __device__ constexpr size_t plane_inv_smem(int S, int NLY, int NLZ, bool acc) {
  return plane_fwd_smem<R>(S, NLY, NLZ) + (acc ? (size_t)S * S * sizeof(R) : 0);
}

// y transforms of columns 0 .. s/2 - 1 of the plane [y][kz], NLY at a time,
// in place.
template <typename C, int S, int NLY>
__device__ __forceinline__ void plane_y_pass(C* plane, C* A, C* B, const C* tw, int dir) {
  constexpr int H = S / 2 + 1;
  for (int q0 = 0; q0 < S / 2; q0 += NLY) {
    auto load = [&](int t, int l) -> C { return plane[t * H + q0 + l]; };
    auto store = [&](int t, int l, C v) { plane[t * H + q0 + l] = v; };
    fft_lines<C, S, NLY, false>(A, B, tw, dir, load, store);
  }
}

// Forward: real plane -> half-spectrum plane, R2C along z and C2C along y.
// a.in, a.out, a.pro (PRO_NONE or PRO_TAPER), a.part as for k_z_r2c; the
// plane index is blockIdx.x.
template <typename R, int S, int NLY, int NLZ, int PRO>
__global__ void __launch_bounds__(kPlaneThreads) k_plane_fwd(ZArgs<R> a) {
  pdl_wait();
  using C = typename Cx<R>::T;
  constexpr int M = S / 2, H = M + 1;
  constexpr int TILE = (int)plane_tile<R>(S, NLY, NLZ);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* plane = reinterpret_cast<C*>(smem_raw);  // [y][kz]; first the real plane [y][z]
  const R* realP = reinterpret_cast<const R*>(smem_raw);
  C* A = plane + S * H;
  C* B = A + TILE;
  C* tw_s = B + TILE;
  C* tw_n = tw_s + S;
  C* tw_m = tw_n + S;
  __shared__ unsigned long long bar;
  const int xi = blockIdx.x;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) tma_load_1d(plane, a.in + (long)xi * S * S, (unsigned)(S * S * sizeof(R)), &bar);
  for (int i = threadIdx.x; i < S; i += blockDim.x) { tw_s[i] = a.tw_s[i]; tw_n[i] = a.tw_n[i]; }
  for (int i = threadIdx.x; i < M; i += blockDim.x) tw_m[i] = a.tw_m[i];
  double shift = 0.0;  // no shell points: no shift
  if constexpr (PRO == PRO_TAPER) {
    if (*a.vmax != 0ull) shift = from_ordered_bits(*a.vmax);
  }
  const bool ok = __syncthreads_and(mbar_wait(&bar, 0, a.err)) != 0;
  if (!ok) return;
  double rowsum = 0.0;
  // R2C along z, NLZ rows at a time, in place: groups run from the last rows
  // down, so a group's complex rows (H complex each) never reach the real
  // rows (S reals each) of the groups still to come
  for (int y0 = S - NLZ; y0 >= 0; y0 -= NLZ) {
    auto load = [&](int m, int l) -> C {
      const int y = y0 + l;
      R x0 = realP[y * S + 2 * m], x1 = realP[y * S + 2 * m + 1];
      if constexpr (PRO == PRO_TAPER) {
        const double h = -0.5 * a.g.L, dx = a.g.dx;
        const double px = h + dx * xi, py = h + dx * y;
        x0 = taper_xyz<R>(a, px, py, h + dx * (2 * m), x0, shift);
        x1 = taper_xyz<R>(a, px, py, h + dx * (2 * m + 1), x1, shift);
      }
      rowsum += (double)x0 + (double)x1;
      return C{x0, x1};
    };
    auto store = [&](int m, int l, C v) { plane[(y0 + l) * H + m] = v; };
    fft_lines<C, M, NLZ, true>(A, B, tw_m, -1, load, store);
    // split Z_q -> X_q = E_q + e^{-2 pi i q/s} O_q, pairs (q, M - q) in place
    for (int w = threadIdx.x; w < (M / 2 + 1) * NLZ; w += blockDim.x) {
      const int l = w / (M / 2 + 1), q = w % (M / 2 + 1);
      C* row = plane + (y0 + l) * H;
      const C zq = row[q], zr = row[(M - q) % M];
      auto split = [&](C za, C zb, int k) -> C {  // X_k from Z_k = za, Z_{M-k} = zb
        const C zc = cconj(zb);
        const C E = cscale(cadd(za, zc), R(0.5));
        const C D = csub(za, zc);  // 2 i O_k
        const C O = {D.y * R(0.5), -D.x * R(0.5)};
        return cadd(E, cmul(tw_n[k], O));
      };
      if (q == 0) {
        const C x0 = split(zq, zq, 0), xm = split(zq, zq, M);
        row[0] = C{x0.x, xm.x};  // X_0 and X_M are real: packed as one column
      } else {
        const C xa = split(zq, zr, q), xb = split(zr, zq, M - q);
        row[q] = xa;
        row[M - q] = xb;
      }
    }
    __syncthreads();
  }
  plane_y_pass<C, S, NLY>(plane, A, B, tw_s, -1);
  // unpack column 0: C(k) = Y_0(k) + i Y_M(k), Y_0 and Y_M Hermitian in k
  for (int k = threadIdx.x; k <= S / 2; k += blockDim.x) {
    const int kr = (S - k) % S;
    const C c = plane[k * H], cr = plane[kr * H];
    const C y0k = {R(0.5) * (c.x + cr.x), R(0.5) * (c.y - cr.y)};
    const C ymk = {R(0.5) * (c.y + cr.y), R(0.5) * (cr.x - c.x)};
    const C y0r = cconj(y0k), ymr = cconj(ymk);
    plane[k * H] = y0k;
    plane[k * H + M] = ymk;
    if (kr != k) {
      plane[kr * H] = y0r;
      plane[kr * H + M] = ymr;
    }
  }
  if (a.part) {
    double acc[1] = {rowsum};
    block_reduce_store<1>(acc, a.part + blockIdx.x);
  }
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) tma_store_1d(a.out + (long)xi * S * H, plane, (unsigned)(S * H * sizeof(C)));
}

// Inverse: a.nin half-spectrum planes -> real outputs with a.epi (as
// k_z_c2r: EPI_GRAD sums the squares of fields 0 .. nin-2 into rout[0] and
// writes field nin-1 to rout[1]; the others write rout[0]).
// EPI is the epilogue a.epi as a template argument: each instantiation
// carries only its own epilogue code, which the last FFT stage inlines once
// per radix output (the instruction cache misses of one kernel holding all
// epilogues were the largest stall).
template <typename R, int S, int NLY, int NLZ, int EPI>
__global__ void __launch_bounds__(kPlaneThreads) k_plane_inv(ZArgs<R> a) {
  pdl_wait();
  using C = typename Cx<R>::T;
  constexpr int M = S / 2, H = M + 1;
  constexpr int TILE = (int)plane_tile<R>(S, NLY, NLZ);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* plane = reinterpret_cast<C*>(smem_raw);  // [y][kz]
  C* A = plane + S * H;
  C* B = A + TILE;
  C* tw_s = B + TILE;
  C* tw_n = tw_s + S;
  C* tw_m = tw_n + S;
  R* acc = reinterpret_cast<R*>(tw_m + M);  // [y][z] (EPI_GRAD); the epilogue tile (Coulomb epilogues)
  __shared__ unsigned long long bar;
  __shared__ double s_f0[kPlaneThreads / 32];
  const int xi = blockIdx.x;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  for (int i = threadIdx.x; i < S; i += blockDim.x) { tw_s[i] = a.tw_s[i]; tw_n[i] = a.tw_n[i]; }
  for (int i = threadIdx.x; i < M; i += blockDim.x) tw_m[i] = a.tw_m[i];
  constexpr bool coul = EPI == EPI_COULOMB || EPI == EPI_COULOMB_V;
  constexpr bool fusev = EPI == EPI_COULOMB_V;
  // V assembly: skipped once the SC loop has exited (V stays as it was)
  const bool vwrite = fusev && !__ldcg(&a.st->exit_loop);
  const double vfac = fusev ? fmin(1.0, __ldcg(&a.st->inc_v)) : 0.0;
  double vacc = 0.0, vmx = -1.0e300;
  double f0 = 0.0;
  if (coul) {  // f0 = dvol * sum of the forward pass's block sums
    double t = 0.0;
    for (int b = threadIdx.x; b < a.f0_blocks; b += blockDim.x) t += a.f0_part[b];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) s_f0[threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (coul) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_f0[w];
    f0 = t * a.g.dvol;
  }
  for (int f = 0; f < a.nin; ++f) {
    if (threadIdx.x == 0) tma_load_1d(plane, a.cin[f] + (long)xi * S * H, (unsigned)(S * H * sizeof(C)), &bar);
    const bool ok = __syncthreads_and(mbar_wait(&bar, (unsigned)(f & 1), a.err)) != 0;
    if (!ok) return;
    // pack columns 0 and M: C(k) = Y_0(k) + i Y_M(k)
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
      const C y0 = plane[k * H], ym = plane[k * H + M];
      plane[k * H] = C{y0.x - ym.y, y0.y + ym.x};
    }
    __syncthreads();
    plane_y_pass<C, S, NLY>(plane, A, B, tw_s, +1);
    // unpack: column 0 holds X_0(y) + i X_M(y), both real
    for (int y = threadIdx.x; y < S; y += blockDim.x) {
      const C c = plane[y * H];
      plane[y * H] = C{c.x, R(0)};
      plane[y * H + M] = C{c.y, R(0)};
    }
    __syncthreads();
    // C2R along z, NLZ rows at a time, with the epilogue
    for (int y0 = 0; y0 < S; y0 += NLZ) {
      auto load = [&](int q, int l) -> C {
        const C* X = plane + (y0 + l) * H;
        const C xq = X[q];
        const C xc = cconj(X[M - q]);
        const C E = cadd(xq, xc);                  // 2 E_q
        const C D = csub(xq, xc);                  // 2 e^{-2 pi i q/s} O_q
        const C O = cmul(cconj(tw_n[q]), D);       // 2 O_q
        return C{E.x - O.y, E.y + O.x};            // 2 (E_q + i O_q)
      };
      auto emit = [&](int m, int l, C z) {
        const int y = y0 + l;
        const R x0 = z.x * R(a.scale), x1 = z.y * R(a.scale);
        const long p0 = ((long)xi * S + y) * S + 2 * m;
        if constexpr (EPI == EPI_GRAD) {
          R* dst = acc + y * S + 2 * m;
          if (f == 0) { dst[0] = x0 * x0; dst[1] = x1 * x1; }
          else if (f < a.nin - 1) { dst[0] += x0 * x0; dst[1] += x1 * x1; }
          else {
            *reinterpret_cast<C*>(a.rout[0] + p0) = C{dst[0], dst[1]};
            *reinterpret_cast<C*>(a.rout[1] + p0) = C{x0, x1};
          }
        } else if constexpr (coul) {
          const double h = -0.5 * a.g.L, dx = a.g.dx;
          const double px = h + dx * xi, py = h + dx * y, pz0 = h + dx * (2 * m), pz1 = h + dx * (2 * m + 1);
          R vh[2];
          if (a.coul_reg) {
            vh[0] = coulomb_xyz<R>(a, px, py, pz0, x0, f0);
            vh[1] = coulomb_xyz<R>(a, px, py, pz1, x1, f0);
          } else {
            vh[0] = R(a.coul_coef * (double)x0);
            vh[1] = R(a.coul_coef * (double)x1);
          }
          *reinterpret_cast<C*>(a.rout[0] + p0) = C{vh[0], vh[1]};
          if (vwrite) {  // k_assemble_v for this point pair (mpDPFT.cpp:4815-4838)
            const C ve = *reinterpret_cast<const C*>(a.vext + p0);
            const C nc = *reinterpret_cast<const C*>(a.ncur + p0);
            const C vo = *reinterpret_cast<const C*>(a.vpot + p0);
            const R vev[2] = {ve.x, ve.y}, ncv[2] = {nc.x, nc.y}, vov[2] = {vo.x, vo.y};
            R vn[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              R vi = vh[i];
              if (a.contact_self) vi += R(2.0 * a.beta) * ncv[i];  // type 10 (:2261)
              if (a.dirac) {                                       // type 11 (:2768)
                R ns = ncv[i] > R(0) ? ncv[i] : R(0);
                vi += R(-a.gamma_h) * cbrt(R(3.0 / kPi) * ns);
              }
              vn[i] = vev[i] + R(vfac) * vi;
              const double d = (double)vn[i] - (double)vov[i];
              vacc += d * d;
              const double pz = i ? pz1 : pz0;
              if (in_shell(px * px + py * py + pz * pz, a.shell_r, a.shell_w)) vmx = fmax(vmx, (double)vn[i]);
            }
            *reinterpret_cast<C*>(a.vpot + p0) = C{vn[0], vn[1]};
          }
        } else if constexpr (EPI == EPI_POS) {
          *reinterpret_cast<C*>(a.rout[0] + p0) = C{x0 > R(0) ? x0 : R(0), x1 > R(0) ? x1 : R(0)};
        } else if constexpr (EPI == EPI_SCALE) {
          *reinterpret_cast<C*>(a.rout[0] + p0) = C{R(a.coul_coef * (double)x0), R(a.coul_coef * (double)x1)};
        } else {
          *reinterpret_cast<C*>(a.rout[0] + p0) = C{x0, x1};
        }
      };
      if constexpr (coul) {
        // the Coulomb epilogues run once per point pair after the transform
        // (from the tile T [l][m], in acc), not inlined at every radix
        // output of its last stage
        C* T = reinterpret_cast<C*>(acc);
        auto store = [&](int m, int l, C z) { T[l * M + m] = z; };
        fft_lines<C, M, NLZ, true>(A, B, tw_m, +1, load, store);
        for (int w = threadIdx.x; w < NLZ * M; w += blockDim.x) emit(w % M, w / M, T[w]);
        __syncthreads();
      } else {
        fft_lines<C, M, NLZ, true>(A, B, tw_m, +1, load, emit);
      }
    }
    // every read of `plane` is done before the next transfer overwrites it
    fence_proxy_async_smem();
    __syncthreads();
  }
  if constexpr (fusev) {  // block sums of |V_new - V_old|^2 and the block's shell maximum
    double accv[1] = {vacc};
    block_reduce_store<1>(accv, a.vres_part + (long)blockIdx.x * kMaxS);
    __shared__ double smx[kPlaneThreads / 32];
    double t = vmx;
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    if ((threadIdx.x & 31) == 0) smx[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = smx[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, smx[w]);
      if (b > -1.0e300) atomicMax(a.vmax_out, ordered_bits(b));
    }
  }
}
