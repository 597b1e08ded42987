// adjoint_kernels.cu -- hand-written adjoint of the time step, for the
// gradient of a trajectory-temperature misfit with respect to the initial
// temperature field.  No counterpart in the reference.
//
// Forward step n (Dirichlet walls, as lb_node_kernel): pull the previous
// post-collision populations (bounce-back / anti-bounce-back at the walls),
// moments rho, j, T with the buoyancy F^n = g*beta rho^{n-1} T^{n-1}, BGK +
// Guo collision, and F^{n+1} = g*beta rho^n T^n.  In the shifted variables
// df_k = f_k - w_k, dg_k = g_k - w_k T0 (the same mathematics as the
// reference-order FP64 arithmetic):
//   dr = sum df, r = 1 + dr, jx = sum cx df, jy = sum cy df
//   u = jx / r,  v = (jy + F/2) / r,  dT = sum dg,  t = T0 + dT
//   cu_k = c_k.u,  P_k = 3 cu + 4.5 cu^2 - 1.5 |u|^2
//   df'_k = (1-w) df_k + w w_k (dr + r P_k) + (1-w/2) w_k F (3 (cy_k - v) + 9 cu_k cy_k)
//   dg'_k = (1-wg) dg_k + wg w_k (dT + t P_k)
//   F' = g*beta r t
// The adjoint kernel of step n, one thread per node x: read the moments the
// forward step formed at x (stored beside the state after the step; they are
// the step's linearisation point) and F^n, apply the transposed local
// Jacobian to the adjoints of the step's outputs at x (lambda df', dg', F',
// plus the observation term on T),
// fold the anti-bounce-back transpose, and push the results to the nodes the
// forward pulled from (the transpose of streaming: bounce-back sends the
// adjoint to the opposite population of the same node; populations that
// stream out of the domain get zero).  Adjoints are FP64.  adjoint_pair_kernel
// runs two such steps per launch through shared memory (see there).
#include <type_traits>

#include "lbrb_internal.cuh"

namespace lbrb {

template <typename Real>
struct AdjView {
  const Real* __restrict__ mom;   // the step's moments as the forward formed them: rho, u, v, T
                                  // planes (the moment planes of the state after the step)
  const Real* __restrict__ Fin;   // F of the step (the state before the step)
  const double* __restrict__ lf_out;  // lambda of the step's post-collision output
  const double* __restrict__ lg_out;
  double* __restrict__ lf_in;     // lambda of the step's input (pushed)
  double* __restrict__ lg_in;
  double* __restrict__ lF;        // in: lambda F^{n+1}; out: lambda F^n (same node)
  long long* __restrict__ lT;     // fixed-point lambda T of this step, or null (read only;
                                  // adj_obs_clear_kernel clears it after the launch)
  int nx, ny, pitch;
  size_t plane;
  double omega, omegag, gbeta, T0, Tup, Tdown;
};

constexpr double ADJ_FIX = 1099511627776.0;  // 2^40

// compile-time loop over the directions
template <int K, typename F>
__device__ __forceinline__ void adj_for(F&& f) {
  if constexpr (K > 0) {
    adj_for<K - 1>(f);
    f(std::integral_constant<int, K - 1>{});
  }
}

// forward quantities of a node at the step: rho, T, u, v and the buoyancy F
struct AdjLoc {
  double r, t, u, v, F;
};

// The step's linearisation point at node offset o: the moments the forward
// step formed there (rho, u, v, T, stored beside the state after the step)
// and the step's buoyancy F.  (Off: element offset type.)
template <typename Real, typename Off = size_t>
__device__ __forceinline__ AdjLoc adj_locals(const Real* __restrict__ mom, const Real* __restrict__ Fin,
                                             size_t plane, Off o) {
  AdjLoc L;
  L.r = (double)mom[o];
  L.u = (double)mom[(Off)plane + o];
  L.v = (double)mom[(Off)(2 * plane) + o];
  L.t = (double)mom[(Off)(3 * plane) + o];
  L.F = (double)Fin[o];
  return L;
}

// weighted moments of 9 adjoint values X_k: sum w_k X_k {1, cx, cy, cx^2,
// cy^2, cx cy}, as tree sums over the D2Q9 directions
struct AdjMom {
  double m0, mx, my, mxx, myy, mxy;
};

template <typename LX>
__device__ __forceinline__ AdjMom adj_moments(LX&& X) {
  constexpr double w0 = w_of(0), w1 = w_of(1), w5 = w_of(5);
  const double s13 = X(1) + X(3), d13 = X(1) - X(3);
  const double s24 = X(2) + X(4), d24 = X(2) - X(4);
  const double c57 = X(5) + X(7), c68 = X(6) + X(8);
  const double e57 = X(5) - X(7), e68 = X(6) - X(8);
  const double cs = c57 + c68;
  AdjMom M;
  M.mxx = fma(w1, s13, w5 * cs);
  M.myy = fma(w1, s24, w5 * cs);
  M.m0 = fma(w0, X(0), fma(w1, s13 + s24, w5 * cs));
  M.mx = fma(w1, d13, w5 * (e57 - e68));
  M.my = fma(w1, d24, w5 * (e57 + e68));
  M.mxy = w5 * (c57 - c68);
  return M;
}

// The adjoint of one step at one node: from the adjoints of the node's
// outputs (post-collision lfo(k), lgo(k); the next step's buoyancy lFo; the
// observation term lt on T) to the adjoints of the values the node pulled
// (outf(k, .), outg(k, .); anti-bounce-back folded in) and of the step's
// buoyancy (lFin).  L: the node's forward quantities at the step.
// The equilibria and the Guo source depend on the populations only through
// rho, u, v (and T), so the transposed Jacobian needs the adjoints only
// through their six weighted moments (M for f, N for g):
//   Phi = om r M + omg t N
//   l_u = 3 Phi_x + 9u Phi_xx + 9v Phi_xy - 3u Phi_0 + 9 s F M_xy
//   l_v = 3 Phi_y + 9u Phi_xy + 9v Phi_yy - 3v Phi_0 + s F (9 M_yy - 3 M_0)
//   Q(X) = X_0 (1 - 1.5|u|^2) + 3(u X_x + v X_y) + 4.5(u^2 X_xx + 2uv X_xy + v^2 X_yy)
//   l_rho = om Q(M) + lFo gb t - (l_u u + l_v v) / r,   l_T = omg Q(N) + lt + lFo gb r
//   l_F = s (3 M_y - 3v M_0 + 9u M_xy + 9v M_yy) + l_v / (2r)
//   out_f_k = (1 - om) lfo_k + l_rho + cx_k l_u / r + cy_k l_v / r
//   out_g_k = (1 - omg) lgo_k + l_T
// with s = 1 - om/2 (om = 1/tau, omg = 1/tau_g, gb = g beta).
template <typename Real, typename LF, typename LG, typename OF, typename OG>
__device__ __forceinline__ void adj_local(const AdjView<Real>& V, const AdjLoc& L, int j, LF&& lfo,
                                          LG&& lgo, double lFo, double lt, OF&& outf, OG&& outg,
                                          double& lFin) {
  const double r = L.r, t = L.t, u = L.u, v = L.v, F = L.F;
  const double rinv = 1.0 / r;
  const double om = V.omega, omg = V.omegag, sf = 1.0 - 0.5 * om;
  const AdjMom M = adj_moments(lfo);
  const AdjMom N = adj_moments(lgo);
  const double al = om * r, be = omg * t;
  const double P0 = fma(al, M.m0, be * N.m0), Px = fma(al, M.mx, be * N.mx);
  const double Py = fma(al, M.my, be * N.my), Pxx = fma(al, M.mxx, be * N.mxx);
  const double Pyy = fma(al, M.myy, be * N.myy), Pxy = fma(al, M.mxy, be * N.mxy);
  const double sF = sf * F;
  // each sum as two independent halves (short dependency chains)
  const double lu = fma(3.0, Px, fma(-3.0 * u, P0, 9.0 * sF * M.mxy)) + fma(9.0 * u, Pxx, 9.0 * v * Pxy);
  const double lv = fma(3.0, Py, fma(-3.0 * v, P0, sF * fma(9.0, M.myy, -3.0 * M.m0))) +
                    fma(9.0 * u, Pxy, 9.0 * v * Pyy);
  const double q15 = 1.0 - 1.5 * fma(u, u, v * v);
  const double uu45 = 4.5 * u * u, vv45 = 4.5 * v * v, uv9 = 9.0 * u * v, u3 = 3.0 * u, v3 = 3.0 * v;
  auto Q = [&](const AdjMom& X) {
    return fma(X.m0, q15, fma(u3, X.mx, v3 * X.my)) + fma(uu45, X.mxx, fma(uv9, X.mxy, vv45 * X.myy));
  };
  const double ldr = fma(om, Q(M), fma(lFo * V.gbeta, t, -fma(lu, u, lv * v) * rinv));
  const double ldT = fma(omg, Q(N), fma(lFo * V.gbeta, r, lt));
  lFin = fma(sf, fma(3.0, M.my, fma(-v3, M.m0, fma(9.0 * u, M.mxy, 9.0 * v * M.myy))), 0.5 * lv * rinv);
  const double ljx = lu * rinv, ljy = lv * rinv;
  // outputs
  double lgs[NPOP];
  adj_for<NPOP>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr int cx = icx(k), cy = icy(k);
    double o = fma(1.0 - om, lfo(k), ldr);
    if constexpr (cx == 1) o += ljx;
    if constexpr (cx == -1) o -= ljx;
    if constexpr (cy == 1) o += ljy;
    if constexpr (cy == -1) o -= ljy;
    outf(k, o);
    lgs[k] = fma(1.0 - omg, lgo(k), ldT);
  });
  // anti-bounce-back transpose: the replaced population feeds its opposite
  if (j == V.ny - 1) {
    lgs[2] -= lgs[4]; lgs[4] = 0.0;
    lgs[5] -= lgs[7]; lgs[7] = 0.0;
    lgs[6] -= lgs[8]; lgs[8] = 0.0;
  }
  if (j == 0) {
    lgs[4] -= lgs[2]; lgs[2] = 0.0;
    lgs[7] -= lgs[5]; lgs[5] = 0.0;
    lgs[8] -= lgs[6]; lgs[6] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < NPOP; k++) outg(k, lgs[k]);
}

// transpose of the pull for one direction: the node's pulled adjoint of
// population k goes to the node the forward pulled it from (bounce-back:
// this node's opposite population; g streaming out of the domain gets zero).
// Every (population, node) of the output receives exactly one write.
template <typename Off = size_t>
__device__ __forceinline__ void adj_push_one(int k, bool is_g, double val, int nx, int ny, int pitch,
                                             size_t plane, int j, int x, double* __restrict__ out) {
  const int xs = icx(k) == 1 ? (x == 0 ? nx - 1 : x - 1) : (icx(k) == -1 ? (x == nx - 1 ? 0 : x + 1) : x);
  const int js = j - icy(k);
  if (js < 0 || js >= ny) out[(Off)opp(k) * (Off)plane + (Off)j * (Off)pitch + (Off)x] = is_g ? 0.0 : val;
  else out[(Off)k * (Off)plane + (Off)js * (Off)pitch + (Off)xs] = val;
}

template <typename Real>
__global__ void __launch_bounds__(128) adjoint_step_kernel(const AdjView<Real> V) {
  pdl_wait();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (x >= V.nx) return;
  const size_t o = (size_t)j * V.pitch + x;
  // every load of the node issued before the arithmetic
  double lf[NPOP], lg[NPOP];
#pragma unroll
  for (int k = 0; k < NPOP; k++) {
    lf[k] = V.lf_out[(size_t)k * V.plane + o];
    lg[k] = V.lg_out[(size_t)k * V.plane + o];
  }
  const double lFo = V.lF[o];
  const double lt = V.lT ? (double)V.lT[o] * (1.0 / ADJ_FIX) : 0.0;
  const AdjLoc L = adj_locals(V.mom, V.Fin, V.plane, o);
  double lFin;
  adj_local(
      V, L, j, [&](int k) { return lf[k]; }, [&](int k) { return lg[k]; }, lFo, lt,
      [&](int k, double val) { adj_push_one(k, false, val, V.nx, V.ny, V.pitch, V.plane, j, x, V.lf_in); },
      [&](int k, double val) { adj_push_one(k, true, val, V.nx, V.ny, V.pitch, V.plane, j, x, V.lg_in); },
      lFin);
  V.lF[o] = lFin;
}

// Two adjoint steps (n, then n-1) in one launch.  A block owns a TX x TY
// tile.  Phase 1 computes step n's pulled adjoints (18 values and lambda F^n)
// at the tile and a one-node ring around it, from lambda^n in HBM, into
// shared memory.  Phase 2 gathers step n-1's output adjoints of each tile
// node from shared memory -- the value the push of step n would have written
// there -- and pushes step n-1's pulled adjoints to lambda^{n-2} in HBM.  The
// FP64 lambda crosses HBM once per two steps instead of once per step.
// lambda F is read from lF (step n+1) and written to lF_out (step n-1), and
// the observation terms lT_a (step n) and lT_b (step n-1) are only read
// (cleared afterwards), since neighbouring blocks read the ring nodes too.
template <typename Real>
struct AdjPairView {
  AdjView<Real> a;                      // step n: its moments and F, lambda^n, lambda F^{n+1}, lambda T^n
  const Real* __restrict__ mom_b;       // moments of step n-1
  const Real* __restrict__ Fin_b;       // F of step n-1
  const long long* __restrict__ lT_b;   // lambda T^{n-1} or null
  double* __restrict__ lf_in;           // lambda^{n-2}
  double* __restrict__ lg_in;
  double* __restrict__ lF_out;          // lambda F^{n-1}
};

// TX x TY tile, NT threads; the ring of (TX+2)(TY+2) nodes takes a second,
// partial round of phase 1 when it has more nodes than the block threads
// (tiles with (TX+2)(TY+2) == NT, e.g. 30x6 on 256 threads, measured slower
// on B200: unaligned rows and more blocks)
template <typename Real, int TX, int TY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) adjoint_pair_kernel(const AdjPairView<Real> P) {
  pdl_wait();
  extern __shared__ double sm[];
  constexpr int HX = TX + 2, HY = TY + 2, NH = HX * HY;
  static_assert(NT >= TX * TY, "one thread per tile node");
  const AdjView<Real>& V = P.a;
  const int nx = V.nx, ny = V.ny;
  const int x0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  // the forward quantities of this thread's phase-2 node do not depend on
  // phase 1: their loads go out first and overlap it
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int x = x0 + tx, j = j0 + ty;
  const bool mine = (int)threadIdx.x < TX * TY && x < nx && j < ny;
  AdjLoc L2{};
  double lt2 = 0.0;
  if (mine) {
    L2 = adj_locals(P.mom_b, P.Fin_b, V.plane, (size_t)j * V.pitch + x);
    if (P.lT_b) lt2 = (double)P.lT_b[(size_t)j * V.pitch + x] * (1.0 / ADJ_FIX);
  }
  // phase 1: step n at the tile and its ring
  for (int h = threadIdx.x; h < NH; h += blockDim.x) {
    const int hx = h % HX, hy = h / HX;
    int xh = x0 - 1 + hx;
    const int jh = j0 - 1 + hy;
    if (xh == -1) xh = nx - 1;
    else if (xh == nx) xh = 0;
    if (jh < 0 || jh >= ny || xh >= nx) continue;  // no node there
    const size_t o = (size_t)jh * V.pitch + xh;
    double lf[NPOP], lg[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      lf[k] = V.lf_out[(size_t)k * V.plane + o];
      lg[k] = V.lg_out[(size_t)k * V.plane + o];
    }
    const double lFo = V.lF[o];
    const double lt = V.lT ? (double)V.lT[o] * (1.0 / ADJ_FIX) : 0.0;
    const AdjLoc L = adj_locals(V.mom, V.Fin, V.plane, o);
    double lFin;
    adj_local(
        V, L, jh, [&](int k) { return lf[k]; }, [&](int k) { return lg[k]; }, lFo, lt,
        [&](int k, double val) { sm[k * NH + h] = val; },
        [&](int k, double val) { sm[(NPOP + k) * NH + h] = val; }, lFin);
    sm[2 * NPOP * NH + h] = lFin;
  }
  __syncthreads();
  // phase 2: step n-1 at the tile
  if (!mine) return;
  const int hs = (tx + 1) + (ty + 1) * HX;  // this node in the ring layout
  // output m of step n-1 at this node went to node (x, j) + c_m (pulled there
  // by step n); at a wall it was bounced back into opp(m) here (f) or left
  // the domain (g)
  auto lfo = [&](int m) {
    const int sj = j + icy(m);
    return (sj < 0 || sj >= ny) ? sm[opp(m) * NH + hs] : sm[m * NH + hs + icx(m) + icy(m) * HX];
  };
  auto lgo = [&](int m) {
    const int sj = j + icy(m);
    return (sj < 0 || sj >= ny) ? 0.0 : sm[(NPOP + m) * NH + hs + icx(m) + icy(m) * HX];
  };
  const size_t o = (size_t)j * V.pitch + x;
  double lFin;
  adj_local(
      V, L2, j, lfo, lgo, sm[2 * NPOP * NH + hs], lt2,
      [&](int k, double val) { adj_push_one(k, false, val, nx, ny, V.pitch, V.plane, j, x, P.lf_in); },
      [&](int k, double val) { adj_push_one(k, true, val, nx, ny, V.pitch, V.plane, j, x, P.lg_in); },
      lFin);
  P.lF_out[o] = lFin;
}

// Marching form of the two steps.  The domain is cut into strips of 32
// columns and groups of RB rows; a unit is one (strip, group).  Block b walks
// down strip b % nstrips over one chunk of `chunk` consecutive groups (chunk
// b / nstrips): the blocks of one chunk run together on neighbouring strips,
// so the halo columns and the pushes across strip edges meet in L2.
// Per unit, phase 1 computes step n's pulled adjoints of the group's next RB
// rows (rows r+1 .. r+RB, 34 columns with the two halo columns) into a ring
// of 2 RB + 2 rows in shared memory, and phase 2 computes step n-1 at rows
// r .. r+RB-1 from the ring.  Rows r-1 and r come from the previous unit, or
// from a prologue step (phase 1 alone, those two rows) where a run starts.
// Phase 1 of one unit writes ring rows that phase 2 of the previous unit
// does not read, so one barrier per unit orders them.  Each thread loads the
// next unit's inputs (lambda^n and the state of its phase-1 node, the state
// of its phase-2 node) into registers before computing the current unit, so
// the loads are in flight during the FP64 arithmetic.  Results are those of
// two adjoint_step_kernel launches, bit for bit.
template <typename Real>
struct MarchIn {
  double lf[NPOP], lg[NPOP], lFo;  // lambda^n and lambda F^{n+1} at the phase-1 node
  long long lt;                    // lambda T^n (fixed point)
  Real ma[4], Fa;                  // moments (rho, u, v, T) and F of step n at the phase-1 node
  Real mb[4], Fb;                  // moments and F of step n-1 at the phase-2 node
  long long ltb;                   // lambda T^{n-1}
};

template <int RB>
struct MarchStep {
  int u;     // unit
  bool pro;  // prologue: phase 1 of rows r-1, r only
};

// PRE = 1: the next unit's inputs go to registers before the current unit's
// arithmetic; PRE = 2: half a unit ahead (phase 2's inputs during phase 1,
// the next phase 1's during phase 2), which holds fewer registers.
template <typename Real, int RB, int MINB, int PRE, typename Off>
__global__ void __launch_bounds__(34 * RB, MINB) adjoint_march_kernel(const AdjPairView<Real> P, int chunk) {
  pdl_wait();
  extern __shared__ double sm[];
  constexpr int HX = 34, S = 2 * RB + 2;  // ring: S rows of HX columns, 2*NPOP+1 values
  const AdjView<Real>& V = P.a;
  const int nx = V.nx, ny = V.ny, pitch = V.pitch;
  const size_t plane = V.plane;
  const int ngroups = (ny + RB - 1) / RB;
  const int nstrips = (nx + 31) / 32;
  const int g0 = (blockIdx.x / nstrips) * chunk;
  const int ub = (blockIdx.x % nstrips) * ngroups + g0;
  const int ue = ub + min(chunk, ngroups - g0);
  if (g0 >= ngroups) return;
  const int t = threadIdx.x;
  const int hx = t % HX, hy = t / HX;  // phase-1 node in the group
  const int px = t % 32, py = t / 32;  // phase-2 node in the group
  auto ring = [&](int v, int row, int col) -> double& { return sm[(v * S + row % S) * HX + col]; };
  // node coordinates of a step for this thread (phase 1: xh, j1; phase 2: x2, j2)
  auto coords = [&](const MarchStep<RB>& st, int& xh, int& j1, bool& a1, int& x2, int& j2, bool& a2) {
    const int s = st.u / ngroups, r = (st.u % ngroups) * RB, x0 = 32 * s;
    j1 = (st.pro ? r - RB : r) + 1 + hy;
    xh = x0 - 1 + hx;
    if (xh == -1) xh = nx - 1;
    else if (xh == nx) xh = 0;
    a1 = j1 >= 0 && j1 < ny && xh < nx && (!st.pro || hy >= RB - 2);
    j2 = r + py;
    x2 = x0 + px;
    a2 = !st.pro && t < 32 * RB && j2 < ny && x2 < nx;
  };
  // inputs of phase 1 (lambda^n and the state before step n at xh, j1) and
  // of phase 2 (the state before step n-1 at x2, j2)
  auto load1 = [&](int xh, int j1, MarchIn<Real>& in) {
    const Off o = (Off)j1 * (Off)pitch + (Off)xh;
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      in.lf[k] = V.lf_out[(Off)k * (Off)plane + o];
      in.lg[k] = V.lg_out[(Off)k * (Off)plane + o];
    }
    in.lFo = V.lF[o];
    in.lt = V.lT ? V.lT[o] : 0ll;
#pragma unroll
    for (int q = 0; q < 4; q++) in.ma[q] = V.mom[(Off)q * (Off)plane + o];
    in.Fa = V.Fin[o];
  };
  auto load2 = [&](int x2, int j2, MarchIn<Real>& in) {
    const Off o = (Off)j2 * (Off)pitch + (Off)x2;
#pragma unroll
    for (int q = 0; q < 4; q++) in.mb[q] = P.mom_b[(Off)q * (Off)plane + o];
    in.Fb = P.Fin_b[o];
    in.ltb = P.lT_b ? P.lT_b[o] : 0ll;
  };
  auto load = [&](const MarchStep<RB>& st, MarchIn<Real>& in) {
    int xh, j1, x2, j2;
    bool a1, a2;
    coords(st, xh, j1, a1, x2, j2, a2);
    if (a1) load1(xh, j1, in);
    if (a2) load2(x2, j2, in);
  };
  auto next = [&](const MarchStep<RB>& st) {
    if (st.pro) return MarchStep<RB>{st.u, false};
    return MarchStep<RB>{st.u + 1, (st.u + 1) % ngroups == 0};  // a new strip starts with a prologue
  };
  auto phase1 = [&](int j1, const MarchIn<Real>& cur) {
    const AdjLoc L{(double)cur.ma[0], (double)cur.ma[3], (double)cur.ma[1], (double)cur.ma[2], (double)cur.Fa};
    double lFin;
    adj_local(
        V, L, j1, [&](int k) { return cur.lf[k]; }, [&](int k) { return cur.lg[k]; }, cur.lFo,
        (double)cur.lt * (1.0 / ADJ_FIX), [&](int k, double val) { ring(k, j1, hx) = val; },
        [&](int k, double val) { ring(NPOP + k, j1, hx) = val; }, lFin);
    ring(2 * NPOP, j1, hx) = lFin;
  };
  auto phase2 = [&](int j2, int x2, const MarchIn<Real>& cur) {
    // output m of step n-1 at this node went to node (x2, j2) + c_m; at a
    // wall it was bounced back into opp(m) here (f) or left the domain (g)
    const int c = px + 1;
    auto lfo = [&](int m) {
      const int sj = j2 + icy(m);
      return (sj < 0 || sj >= ny) ? ring(opp(m), j2, c) : ring(m, sj, c + icx(m));
    };
    auto lgo = [&](int m) {
      const int sj = j2 + icy(m);
      return (sj < 0 || sj >= ny) ? 0.0 : ring(NPOP + m, sj, c + icx(m));
    };
    const AdjLoc L{(double)cur.mb[0], (double)cur.mb[3], (double)cur.mb[1], (double)cur.mb[2], (double)cur.Fb};
    double lFin;
    adj_local(
        V, L, j2, lfo, lgo, ring(2 * NPOP, j2, c), (double)cur.ltb * (1.0 / ADJ_FIX),
        [&](int k, double val) { adj_push_one<Off>(k, false, val, nx, ny, pitch, plane, j2, x2, P.lf_in); },
        [&](int k, double val) { adj_push_one<Off>(k, true, val, nx, ny, pitch, plane, j2, x2, P.lg_in); },
        lFin);
    P.lF_out[(Off)j2 * (Off)pitch + (Off)x2] = lFin;
  };
  auto compute = [&](const MarchStep<RB>& st, const MarchIn<Real>& cur) {
    int xh, j1, x2, j2;
    bool a1, a2;
    coords(st, xh, j1, a1, x2, j2, a2);
    // a prologue inside the run: the previous unit's phase 2 may still read
    // the ring rows it writes
    if (st.pro && st.u != ub) __syncthreads();
    if (a1) phase1(j1, cur);
    if (!st.pro) {
      __syncthreads();
      if (a2) phase2(j2, x2, cur);
    }
  };
  MarchStep<RB> st{ub, true};
  if constexpr (PRE == 1) {
    // the next step's loads go out before the current step's arithmetic
    MarchIn<Real> cur;
    load(st, cur);
    for (;;) {
      const MarchStep<RB> nst = next(st);
      const bool more = nst.u < ue;
      MarchIn<Real> nxt;
      if (more) load(nst, nxt);
      compute(st, cur);
      if (!more) break;
      cur = nxt;
      st = nst;
    }
  } else {
    static_assert(PRE == 2, "prefetch form");
    // half a step ahead: phase 2's loads go out before phase 1's arithmetic,
    // the next step's phase-1 loads before phase 2's arithmetic
    MarchIn<Real> in1, in2;
    int xh, j1, x2, j2;
    bool a1, a2;
    coords(st, xh, j1, a1, x2, j2, a2);
    if (a1) load1(xh, j1, in1);
    for (;;) {
      if (a2) load2(x2, j2, in2);
      if (st.pro && st.u != ub) __syncthreads();
      if (a1) phase1(j1, in1);
      const MarchStep<RB> nst = next(st);
      const bool more = nst.u < ue;
      int nxh, nj1, nx2, nj2;
      bool na1 = false, na2 = false;
      if (more) {
        coords(nst, nxh, nj1, na1, nx2, nj2, na2);
        if (na1) load1(nxh, nj1, in1);
      }
      if (!st.pro) {
        __syncthreads();
        if (a2) phase2(j2, x2, in2);
      }
      if (!more) break;
      st = nst;
      xh = nxh, j1 = nj1, a1 = na1, x2 = nx2, j2 = nj2, a2 = na2;
    }
  }
}

// observation adjoint of step n: lambda T += 2 r_p w_corner, fixed point
__global__ void adj_obs_scatter_kernel(const double* __restrict__ ox, const double* __restrict__ oy,
                                       const double* __restrict__ res, int nobs, int nx, int ny,
                                       int pitch, unsigned long long* __restrict__ acc) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  const double xx = ox[p], yy = oy[p];
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) return;
  const int x1 = (int)xx, y1 = (int)yy, x2 = x1 + 1, y2 = y1 + 1;
  int ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  int ix2 = (x2 - 1) % nx; if (ix2 < 0) ix2 += nx;
  int jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  int jy2 = (y2 - 1) % ny; if (jy2 < 0) jy2 += ny;
  const double g = 2.0 * res[p];
  const double wx1 = (double)x2 - xx, wx2 = xx - (double)x1;
  const double wy1 = (double)y2 - yy, wy2 = yy - (double)y1;
  atomicAdd(&acc[(size_t)jy1 * pitch + ix1], (unsigned long long)__double2ll_rn(g * wx1 * wy1 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy1 * pitch + ix2], (unsigned long long)__double2ll_rn(g * wx2 * wy1 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy2 * pitch + ix1], (unsigned long long)__double2ll_rn(g * wx1 * wy2 * ADJ_FIX));
  atomicAdd(&acc[(size_t)jy2 * pitch + ix2], (unsigned long long)__double2ll_rn(g * wx2 * wy2 * ADJ_FIX));
}

// residuals r_p = T(x_p) - T_obs,p of one observation step (forward)
template <typename Real>
__global__ void obs_residual_kernel(const Real* __restrict__ T, int nx, int ny, int pitch,
                                    const double* __restrict__ ox, const double* __restrict__ oy,
                                    const double* __restrict__ oT, int nobs, double* __restrict__ res) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  const double xx = ox[p], yy = oy[p];
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) { res[p] = 0.0; return; }
  const int x1 = (int)xx, y1 = (int)yy, x2 = x1 + 1, y2 = y1 + 1;
  int ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  int ix2 = (x2 - 1) % nx; if (ix2 < 0) ix2 += nx;
  int jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  int jy2 = (y2 - 1) % ny; if (jy2 < 0) jy2 += ny;
  const double u11 = (double)T[(size_t)jy1 * pitch + ix1], u12 = (double)T[(size_t)jy2 * pitch + ix1];
  const double u21 = (double)T[(size_t)jy1 * pitch + ix2], u22 = (double)T[(size_t)jy2 * pitch + ix2];
  const double tm = u11 * ((double)x2 - xx) * ((double)y2 - yy) + u21 * (xx - (double)x1) * ((double)y2 - yy) +
                    u12 * ((double)x2 - xx) * (yy - (double)y1) + u22 * (xx - (double)x1) * (yy - (double)y1);
  res[p] = tm - oT[p];
}

// initial state from a temperature field T0 (f = feq(1,0), g = geq(T0,0),
// moments by the restart route), as lbrb_init_conduction without the profile
template <typename Real>
__global__ void init_from_T0_kernel(const double* __restrict__ T0f, Real* __restrict__ pops,
                                    Real* __restrict__ rho, Real* __restrict__ u, Real* __restrict__ v,
                                    Real* __restrict__ T, Real* __restrict__ F, int nx, int ny,
                                    int pitch, size_t plane, double Tref, double neg_gravity) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    const double t = T0f[q];
    double feq[NPOP], geq[NPOP];
    equil_ref(1.0, 0.0, 0.0, feq);
    equil_ref(t, 0.0, 0.0, geq);
    double r = 0.0, tt = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      r = r + feq[k];
      if constexpr (std::is_same<Real, double>::value) {
        pops[(size_t)k * plane + o] = feq[k];
        pops[(size_t)(k + NPOP) * plane + o] = geq[k];
      } else {
        pops[(size_t)k * plane + o] = (float)(feq[k] - w_of(k));
        pops[(size_t)(k + NPOP) * plane + o] = (float)(geq[k] - w_of(k) * Tref);
      }
    }
#pragma unroll
    for (int k = 0; k < NPOP; k++) tt = tt + geq[k];
    const double rhoi = 1. / r;
    double fl[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; k++) fl[k] = feq[k] * rhoi;
    rho[o] = (Real)r;
    T[o] = (Real)tt;
    u[o] = (Real)(fl[1] - fl[3] + fl[5] - fl[6] - fl[7] + fl[8]);
    v[o] = (Real)(fl[5] + fl[2] + fl[6] - fl[7] - fl[4] - fl[8] + (0.5 * neg_gravity * tt));
    if constexpr (std::is_same<Real, double>::value) F[o] = neg_gravity * r * (tt - 0.0);
    else F[o] = (float)neg_gravity * (float)r * (float)tt;
  }
}

// gradient with respect to T0: sum_k w_k lambda g_k^0 + g*beta rho^0 (sum_k w_k) lambda F^1
__global__ void adj_initial_kernel(const double* __restrict__ lg, const double* __restrict__ lF,
                                   int nx, int ny, int pitch, size_t plane, double gbeta,
                                   double* __restrict__ out) {
  const long n = (long)nx * ny;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)(q / nx);
    const size_t o = (size_t)j * pitch + i;
    double s = 0.0, sw = 0.0, r0 = 0.0, feq[NPOP];
    equil_ref(1.0, 0.0, 0.0, feq);
#pragma unroll
    for (int k = 0; k < NPOP; k++) {
      s += w_of(k) * lg[(size_t)k * plane + o];
      sw += w_of(k);
      r0 = r0 + feq[k];
    }
    out[q] = s + gbeta * r0 * sw * lF[o];
  }
}

// clear the observation adjoint of one step after its consumer kernel ran
// (the corners the scatter touched)
__global__ void adj_obs_clear_kernel(const double* __restrict__ ox, const double* __restrict__ oy,
                                     int nobs, int nx, int ny, int pitch, long long* __restrict__ acc) {
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nobs) return;
  const double xx = ox[p], yy = oy[p];
  if (!(xx > -2.0 && xx < nx + 2.0 && yy > -2.0 && yy < ny + 2.0)) return;
  const int x1 = (int)xx, y1 = (int)yy, x2 = x1 + 1, y2 = y1 + 1;
  int ix1 = (x1 - 1) % nx; if (ix1 < 0) ix1 += nx;
  int ix2 = (x2 - 1) % nx; if (ix2 < 0) ix2 += nx;
  int jy1 = (y1 - 1) % ny; if (jy1 < 0) jy1 += ny;
  int jy2 = (y2 - 1) % ny; if (jy2 < 0) jy2 += ny;
  acc[(size_t)jy1 * pitch + ix1] = 0;
  acc[(size_t)jy1 * pitch + ix2] = 0;
  acc[(size_t)jy2 * pitch + ix1] = 0;
  acc[(size_t)jy2 * pitch + ix2] = 0;
}

// misfit J = sum of squared residuals: per-thread Neumaier sums in a fixed
// order, combined by a tree of error-free additions (deterministic)
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bp = s - a;
  e = (a - (s - bp)) + (b - bp);
}

__global__ void __launch_bounds__(1024) misfit_kernel(const double* __restrict__ res, long n,
                                                      double* __restrict__ out) {
  pdl_wait();
  __shared__ double ss[1024], sc[1024];
  double sum = 0.0, comp = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = res[i] * res[i];
    double t, e;
    two_sum(sum, x, t, e);
    sum = t;
    comp += e;
  }
  ss[threadIdx.x] = sum;
  sc[threadIdx.x] = comp;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      double t, e;
      two_sum(ss[threadIdx.x], ss[threadIdx.x + w], t, e);
      ss[threadIdx.x] = t;
      sc[threadIdx.x] += sc[threadIdx.x + w] + e;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = ss[0] + sc[0];
}

// ---------------------------------------------------------------- launchers
template <typename Real, int TX, int TY, int NT, int MINB>
static cudaError_t launch_pair_t(const AdjPairView<Real>& P, cudaStream_t s) {
  constexpr int NH = (TX + 2) * (TY + 2);
  constexpr size_t smem = (size_t)(2 * NPOP + 1) * NH * sizeof(double);
  static std::atomic<unsigned long long> attr_set{0};
  const cudaError_t attr =
      smem_limit_once((const void*)adjoint_pair_kernel<Real, TX, TY, NT, MINB>, smem, attr_set);
  if (attr != cudaSuccess) return attr;
  dim3 grid((P.a.nx + TX - 1) / TX, (P.a.ny + TY - 1) / TY);
  return launch_k(adjoint_pair_kernel<Real, TX, TY, NT, MINB>, grid, NT, smem, s, true, P);
}

// marching kernel: strips x chunks blocks, the chunk length chosen so that
// the grid fills about `waves` waves of resident blocks
template <typename Real, int RB, int MINB, int PRE, typename Off>
static cudaError_t launch_march_o(const AdjPairView<Real>& P, int waves, cudaStream_t s) {
  constexpr int NT = 34 * RB;
  constexpr size_t smem = (size_t)(2 * NPOP + 1) * (2 * RB + 2) * 34 * sizeof(double);
  auto kern = adjoint_march_kernel<Real, RB, MINB, PRE, Off>;
  static std::atomic<unsigned long long> attr_set{0};
  static std::atomic<int> occ_cache[MAX_DEVICES] = {};
  const cudaError_t attr = smem_limit_once((const void*)kern, smem, attr_set);
  if (attr != cudaSuccess) return attr;
  int occ = 0;
  cudaError_t e = occupancy_once((const void*)kern, NT, smem, occ_cache, &occ);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0;
  e = current_device(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int nstrips = (P.a.nx + 31) / 32, ngroups = (P.a.ny + RB - 1) / RB;
  const int target = std::max(1, nsm * occ * waves / nstrips);  // chunks per strip
  const int chunk = (ngroups + target - 1) / target;
  const int nchunks = (ngroups + chunk - 1) / chunk;
  return launch_k(kern, nstrips * nchunks, NT, smem, s, true, P, chunk);
}

// 32-bit element offsets where 36 planes of the grid fit below 2^32
template <typename Real, int RB, int MINB, int PRE>
static cudaError_t launch_march_t(const AdjPairView<Real>& P, int waves, cudaStream_t s) {
  if (off32_ok(P.a.plane)) return launch_march_o<Real, RB, MINB, PRE, uint32_t>(P, waves, s);
  return launch_march_o<Real, RB, MINB, PRE, size_t>(P, waves, s);
}

// launch variants of the two-step adjoint: 0-3 the tiled pair kernel (tile
// TX x TY, threads, min blocks per SM), 4-9 the marching kernel (rows per
// group, blocks per SM, register prefetch; waves of blocks)
constexpr int ADJ_NPAIR_VARIANTS = 10;
int adjoint_pair_variants() { return ADJ_NPAIR_VARIANTS; }

// steps n and n-1 from the moment blocks (MB_PLANES planes: F, rho, u, v, T)
// of three states: after_a (the state after step n: its moments are step n's
// linearisation point), state_a (before step n: F^n, and its moments are
// step n-1's), state_b (before step n-1: F^{n-1}); lambda^n in (lf_out,
// lg_out), lambda^{n-2} out (lf_in, lg_in), lambda F^{n+1} in (lF_in),
// lambda F^{n-1} out (lF_out)
cudaError_t launch_adjoint_pair(bool fp32, int variant, const void* after_a, const void* state_a,
                                const void* state_b, const double* lf_out, const double* lg_out,
                                double* lf_in, double* lg_in, double* lF_in, double* lF_out,
                                const long long* lT_a, const long long* lT_b, int nx, int ny, int pitch,
                                size_t plane, double omega, double omegag, double gbeta, double T0,
                                double Tup, double Tdown, cudaStream_t s) {
  auto go = [&](auto zero) -> cudaError_t {
    using Real = decltype(zero);
    const Real* n1 = (const Real*)after_a;
    const Real* a = (const Real*)state_a;
    const Real* b = (const Real*)state_b;
    AdjPairView<Real> P{};
    P.a = AdjView<Real>{n1 + plane, a, lf_out, lg_out, nullptr, nullptr,
                        lF_in, const_cast<long long*>(lT_a), nx, ny, pitch, plane, omega, omegag,
                        gbeta, T0, Tup, Tdown};
    P.mom_b = a + plane;
    P.Fin_b = b;
    P.lT_b = lT_b;
    P.lf_in = lf_in;
    P.lg_in = lg_in;
    P.lF_out = lF_out;
    switch (variant) {
      case 1: return launch_pair_t<Real, 32, 4, 128, 6>(P, s);
      case 2: return launch_pair_t<Real, 32, 8, 256, 2>(P, s);
      case 3: return launch_pair_t<Real, 32, 8, 256, 3>(P, s);
      case 4: return launch_march_t<Real, 7, 1, 1>(P, 2, s);
      case 5: return launch_march_t<Real, 6, 1, 1>(P, 2, s);
      case 6: return launch_march_t<Real, 7, 1, 2>(P, 2, s);
      case 7: return launch_march_t<Real, 5, 2, 2>(P, 2, s);
      case 8: return launch_march_t<Real, 5, 2, 2>(P, 1, s);
      case 9: return launch_march_t<Real, 3, 3, 2>(P, 2, s);
      default: return launch_pair_t<Real, 32, 4, 128, 4>(P, s);
    }
  };
  return fp32 ? go(0.f) : go(0.0);
}

template <typename Real>
static cudaError_t launch_adj_t(const AdjView<Real>& V, cudaStream_t s) {
  dim3 grid((V.nx + 127) / 128, V.ny);
  return launch_k(adjoint_step_kernel<Real>, grid, 128, 0, s, true, V);
}

// one step from the moment blocks of two states: `after` (its moments: the
// step's linearisation point) and `state` (before the step: F)
cudaError_t launch_adjoint_step(bool fp32, const void* after, const void* state, const double* lf_out,
                                const double* lg_out, double* lf_in, double* lg_in, double* lF,
                                long long* lT, int nx, int ny, int pitch, size_t plane, double omega,
                                double omegag, double gbeta, double T0, double Tup, double Tdown,
                                cudaStream_t s) {
  if (fp32) {
    AdjView<float> V{(const float*)after + plane, (const float*)state, lf_out,
                     lg_out, lf_in, lg_in, lF, lT, nx, ny, pitch, plane, omega, omegag, gbeta, T0, Tup,
                     Tdown};
    return launch_adj_t(V, s);
  }
  AdjView<double> V{(const double*)after + plane, (const double*)state, lf_out,
                    lg_out, lf_in, lg_in, lF, lT, nx, ny, pitch, plane, omega, omegag, gbeta, T0, Tup,
                    Tdown};
  return launch_adj_t(V, s);
}

cudaError_t launch_misfit(const double* res, long n, double* out, cudaStream_t s) {
  return launch_k(misfit_kernel, 1, 1024, 0, s, true, res, n, out);
}

cudaError_t launch_adj_obs_clear(const double* ox, const double* oy, int nobs, int nx, int ny, int pitch,
                                 long long* acc, cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  return launch_k(adj_obs_clear_kernel, (nobs + 127) / 128, 128, 0, s, true, ox, oy, nobs, nx, ny, pitch, acc);
}

cudaError_t launch_adj_obs_scatter(const double* ox, const double* oy, const double* res, int nobs,
                                   int nx, int ny, int pitch, long long* acc, cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  return launch_k(adj_obs_scatter_kernel, (nobs + 127) / 128, 128, 0, s, true, ox, oy, res, nobs, nx, ny, pitch,
                  reinterpret_cast<unsigned long long*>(acc));
}

cudaError_t launch_obs_residual(const void* T, bool fp32, int nx, int ny, int pitch, const double* ox,
                                const double* oy, const double* oT, int nobs, double* res,
                                cudaStream_t s) {
  if (nobs <= 0) return cudaSuccess;
  if (fp32)
    return launch_k(obs_residual_kernel<float>, (nobs + 127) / 128, 128, 0, s, true, (const float*)T, nx, ny,
                    pitch, ox, oy, oT, nobs, res);
  return launch_k(obs_residual_kernel<double>, (nobs + 127) / 128, 128, 0, s, true, (const double*)T, nx, ny,
                  pitch, ox, oy, oT, nobs, res);
}

cudaError_t launch_init_from_T0(const double* T0f, void* pops, void* rho, void* u, void* v, void* T,
                                void* F, bool fp32, int nx, int ny, int pitch, size_t plane,
                                double Tref, double neg_gravity, cudaStream_t s) {
  const int g = 148 * 8;
  if (fp32)
    init_from_T0_kernel<float><<<g, 256, 0, s>>>(T0f, (float*)pops, (float*)rho, (float*)u, (float*)v,
                                                 (float*)T, (float*)F, nx, ny, pitch, plane, Tref, neg_gravity);
  else
    init_from_T0_kernel<double><<<g, 256, 0, s>>>(T0f, (double*)pops, (double*)rho, (double*)u, (double*)v,
                                                  (double*)T, (double*)F, nx, ny, pitch, plane, Tref, neg_gravity);
  return cudaGetLastError();
}

cudaError_t launch_adj_initial(const double* lg, const double* lF, int nx, int ny, int pitch,
                               size_t plane, double gbeta, double* out, cudaStream_t s) {
  adj_initial_kernel<<<148 * 8, 256, 0, s>>>(lg, lF, nx, ny, pitch, plane, gbeta, out);
  return cudaGetLastError();
}

}  // namespace lbrb
