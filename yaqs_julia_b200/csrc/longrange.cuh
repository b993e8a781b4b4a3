// Long-range noise processes (MPONoiseProcess, Noise.jl:22-33) on sites
// a < b - 1 with operator O = alpha*1 + beta*(sig at a)(tau at b), the MPO of
// build_mpo_phys (Noise.jl:71-131): bond dimension 2 on the bonds a..b-1.
//
// The reference applies O to the state as an MPO, contracting site by site
// (apply_mpo_jump!, StochasticProcess.jl:46-82), and then runs MPS.truncate!
// (MPS.jl:320-440): the centre is moved to site 1 by LQ steps from site L,
// one SVD sweep 1 -> L-1 truncates each bond (absolute rule, min 2, at most
// max_bond_dim), and normalize! renormalises.  Here the same factorisations
// run with the doubled tensors built one at a time from the state:
//  - the LQ walk from L to b+1 is the state's own gauge walk (O acts as the
//    identity there);
//  - sites b..a take the operator's rows and columns and keep their
//    right-canonical factors in the lrQ arena (bonds up to twice the cap);
//  - sites a-1..1 continue in place;
//  - the SVD sweep factorises the centre alone: with the right part
//    right-canonical, the SVD of (centre x next site) has the same singular
//    values and left vectors as the SVD of the centre, and S V^H of the pair
//    is (S V^H of the centre) x next site.
// Candidate weights: the reference weighs an "mpo_general" candidate by the
// norm of its applied, truncated and renormalised copy, which is 1 unless
// the applied operator annihilates the state (norm below 1e-13 before the
// rescale, normalize! at MPS.jl:302-306).  lr_weight computes the norm of
// O|psi> by a QR sweep from site a (orthogonal factorisations keep the
// absolute error near machine precision, so a cancelled branch reads ~1e-16
// as in the reference) and returns 1 or that tiny norm squared.

struct LrBufs {
  cplx *Q, *Phi, *M, *H, *Qh, *Lf, *R, *C0, *C1;
  int* bd;  // [L+1] bond dimensions of the operator-applied chain
};

static __device__ __forceinline__ LrBufs lr_bufs(const Ctx& c) {
  LrBufs b;
  b.Q = c.ws + c.P.lay.lrQ;
  b.Phi = c.ws + c.P.lay.lrPhi;
  b.M = c.ws + c.P.lay.lrM;
  b.H = c.ws + c.P.lay.lrH;
  b.Qh = c.ws + c.P.lay.lrQh;
  b.Lf = c.ws + c.P.lay.lrL;
  b.R = c.ws + c.P.lay.lrR;
  b.C0 = c.ws + c.P.lay.lrC0;
  b.C1 = c.ws + c.P.lay.lrC1;
  b.bd = c.wsi + c.P.lay.i_lr;
  return b;
}

// Right-canonical factor of site k in the lrQ arena (room for twice the
// state's caps on both bonds).
static __device__ __forceinline__ cplx* lr_qslot(const Ctx& c, const LrBufs& b, int k) {
  return b.Q + 4 * c.P.mps_off[k];
}

// Site k of O|psi> as a dense (lo, 2, ro) tensor: the contraction
// C[la, lw, po, ra, rw] of apply_mpo_jump! with (la, lw) and (ra, rw) merged,
// la and ra fastest.  A is the state's tensor (l, 2, r).
static __device__ void lr_phi(const DevProc& pr, int k, const cplx* A, int l, int r, cplx* out, int& lo, int& ro) {
  const int a = pr.s0, b = pr.s1;
  const cplx* sig = pr.mat;
  const cplx* tau = pr.mat + 4;
  const cplx alpha = pr.mat[8], beta = pr.mat[9];
  if (k < a || k > b) {
    lo = l;
    ro = r;
  } else if (k == a) {
    lo = l;
    ro = 2 * r;
  } else if (k < b) {
    lo = 2 * l;
    ro = 2 * r;
  } else {
    lo = 2 * l;
    ro = r;
  }
  const long long n = (long long)lo * 2 * ro;
  for (long long e = ltid(); e < n; e += NT) {
    const int L_ = (int)(e % lo);
    const int p = (int)((e / lo) % 2);
    const int R_ = (int)(e / (2LL * lo));
    const int li = L_ % l, lw = L_ / l, ri = R_ % r, rw = R_ / r;
    const cplx a0 = A[li + (long long)l * (0 + 2LL * ri)];
    const cplx a1 = A[li + (long long)l * (1 + 2LL * ri)];
    const cplx ap = p == 0 ? a0 : a1;
    cplx v = make_double2(0.0, 0.0);
    if (k < a || k > b) {
      v = ap;
    } else if (k == a) {  // row [1, sig]
      v = rw == 0 ? ap : cadd(cmul(sig[p], a0), cmul(sig[p + 2], a1));
    } else if (k < b) {  // diag(1, 1)
      v = lw == rw ? ap : make_double2(0.0, 0.0);
    } else {  // column [alpha 1; beta tau]
      v = lw == 0 ? cmul(alpha, ap) : cmul(beta, cadd(cmul(tau[p], a0), cmul(tau[p + 2], a1)));
    }
    out[e] = v;
  }
  cta_sync();
}

// LQ of M (rows x cols, ld rows) = Lout (rows x rn) Qout (rn x cols),
// rn = min(rows, cols), through the Householder QR of M^H (the factorisation
// lq_left uses).  rows <= SVD_MAX_COLS.
static __device__ int lr_lq(Ctx& c, const LrBufs& b, const cplx* M, int rows, int cols, cplx* Lout, cplx* Qout) {
  const int rn = min(rows, cols);
  for (long long e = ltid(); e < (long long)cols * rows; e += NT) {
    const int cc = (int)(e % cols), ii = (int)(e / cols);
    b.H[e] = cconj(M[ii + (long long)rows * cc]);
  }
  cta_sync();
  dev_qr_factor(b.H, cols, rows, c.sm.la, c.sm.e.r);
  dev_qr_formq(b.H, cols, rows, b.Qh, c.sm.la);
  dev_qr_extract_r(b.H, cols, rows, b.R);  // rn x rows
  for (long long e = ltid(); e < (long long)rn * cols; e += NT) {
    const int k = (int)(e % rn), cc = (int)(e / rn);
    Qout[e] = cconj(b.Qh[cc + (long long)cols * k]);
  }
  for (long long e = ltid(); e < (long long)rows * rn; e += NT) {
    const int i = (int)(e % rows), k = (int)(e / rows);
    Lout[e] = cconj(b.R[k + (long long)rn * i]);
  }
  cta_sync();
  return rn;
}

// Candidate weight factor of an "mpo_general" process (see above): 1 when
// O|psi> is not null, else its (tiny) norm squared.  The state's centre
// sits at site L-1 with sites 0..L-2 left-canonical, so the sweep starts at
// site a with an identity on the left.  Reads the state only.
static __device__ __noinline__ double lr_weight(Ctx& c, const DState& s, const DevProc& pr) {
  const int L = c.P.L;
  LrBufs b = lr_bufs(c);
  int lo, ro;
  int kq = 0;
  double nrm2 = 0.0;
  for (int k = pr.s0; k < L && !c.sm.fail; ++k) {
    lr_phi(pr, k, site_ptr(c, s, k), s.chi[k], s.chi[k + 1], b.Phi, lo, ro);
    int rows;
    if (k == pr.s0) {  // M = Phi as (2 lo) x ro
      cta_copy(b.M, b.Phi, (long long)lo * 2 * ro);
      rows = 2 * lo;
    } else {  // M = R (kq x lo) Phi (lo x 2 ro), viewed as (2 kq) x ro
      cta_gemm(gemm_args(kq, 2 * ro, lo, b.R, 1, kq, b.Phi, 1, lo, b.M, 1, kq), c.sm.e.u.gw.g);
      rows = 2 * kq;
    }
    cta_sync();
    if (k == L - 1) {
      nrm2 = cta_norm2(b.M, (long long)rows * ro, c.sm.e.r);
      break;
    }
    dev_qr_factor(b.M, rows, ro, c.sm.la, c.sm.e.r);
    kq = min(rows, ro);
    dev_qr_extract_r(b.M, rows, ro, b.R);  // kq x ro
  }
  return sqrt(nrm2) > 1e-13 ? 1.0 : nrm2;
}

// apply_mpo_jump! followed by MPS.truncate! (see above).  Expects the
// centre at site L-1; leaves the state normalised with the centre at 0.
static __device__ __noinline__ void lr_apply(Ctx& c, const DState& s, const DevProc& pr) {
  const int L = c.P.L, a = pr.s0, bb = pr.s1;
  LrBufs b = lr_bufs(c);
  // ---- LQ walk L-1 -> 1 of O|psi> ----
  shift_oc(c, s, bb);  // O is the identity right of b
  if (c.sm.fail) return;
  int lo, ro;
  lr_phi(pr, bb, site_ptr(c, s, bb), s.chi[bb], s.chi[bb + 1], b.Phi, lo, ro);
  int rn = lr_lq(c, b, b.Phi, lo, 2 * ro, b.Lf, lr_qslot(c, b, bb));
  if (ltid() == 0) {
    b.bd[bb] = rn;
    for (int k = bb + 1; k <= L; ++k) b.bd[k] = s.chi[k];
  }
  int lf_rows = lo, lf_cols = rn;
  cplx* C = b.C0;
  bool centre_done = false;
  for (int k = bb - 1; k >= a && !c.sm.fail; --k) {
    lr_phi(pr, k, site_ptr(c, s, k), s.chi[k], s.chi[k + 1], b.Phi, lo, ro);  // ro == lf_rows
    cta_gemm(gemm_args(2 * lo, lf_cols, ro, b.Phi, 1, 2 * lo, b.Lf, 1, lf_rows, b.M, 1, 2 * lo), c.sm.e.u.gw.g);
    cta_sync();
    if (k == 0) {  // site 0 is never factorised: it is the centre
      cta_copy(C, b.M, (long long)lo * 2 * lf_cols);
      if (ltid() == 0) {
        b.bd[0] = lo;
        b.bd[1] = lf_cols;
      }
      centre_done = true;
      break;
    }
    rn = lr_lq(c, b, b.M, lo, 2 * lf_cols, b.Lf, lr_qslot(c, b, k));
    if (ltid() == 0) b.bd[k] = rn;
    lf_rows = lo;
    lf_cols = rn;
  }
  if (c.sm.fail) return;
  if (!centre_done) {
    // absorb the last L factor into site a-1 (in place), then the state's own walk to site 0
    const int lp = s.chi[a - 1];
    cplx* Ap = site_ptr(c, s, a - 1);
    cta_gemm(gemm_args(2 * lp, lf_cols, lf_rows, Ap, 1, 2 * lp, b.Lf, 1, lf_rows, b.M, 1, 2 * lp), c.sm.e.u.gw.g);
    cta_sync();
    cta_copy(Ap, b.M, (long long)2 * lp * lf_cols);
    set_chi(c, s, a, lf_cols);
    for (int i = a - 1; i >= 1 && !c.sm.fail; --i) lq_left(c, s, i);
    if (c.sm.fail) return;
    cta_copy(C, site_ptr(c, s, 0), (long long)s.chi[0] * 2 * s.chi[1]);
    if (ltid() == 0)
      for (int k = 0; k <= a; ++k) b.bd[k] = s.chi[k];
  }
  cta_sync();
  // ---- SVD sweep 0 -> L-2 (absolute rule, min 2, at most max_bond) ----
  cplx* Cn = b.C1;
  for (int k = 0; k + 1 < L && !c.sm.fail; ++k) {
    const int l = b.bd[k], r = b.bd[k + 1], r2 = b.bd[k + 2];
    const int m = 2 * l;
    SvdWork w = svd_work(c);
    SvdResult res = dev_svd(C, m, r, SVD_LEFT, w, c.sm.la, c.sm.e.r, c.sm.e.u.svd);
    if (ltid() == 0) {
      c.sm.bcast_i[0] = keep_tdvp(w.sig, res.p, c.P.thr, c.P.max_bond);
      c.cnt[2] += 1;
      c.cnt[5] += res.sweeps;
    }
    cta_sync();
    const int keep = c.sm.bcast_i[0];
    cta_sync();
    if (keep > c.P.cap[k + 1]) {
      if (ltid() == 0) c.sm.fail = ST_UNSUPPORTED;
      cta_sync();
      return;
    }
    dev_svd_vectors(res, keep, w, c.sm.e.r);
    cta_copy(site_ptr(c, s, k), w.Yo, (long long)m * keep);
    // S V^H = U^H C (keep x r), rows past the rank exactly zero
    cta_gemm(gemm_args(keep, r, m, w.Yo, m, 1, C, 1, m, b.R, 1, keep, true, false), c.sm.e.u.gw.g);
    cta_sync();
    for (int e = ltid(); e < keep * r; e += NT)
      if ((e % keep) >= res.rank) b.R[e] = make_double2(0.0, 0.0);
    cta_sync();
    const cplx* Bn = (k + 1 >= a && k + 1 <= bb) ? lr_qslot(c, b, k + 1) : site_ptr(c, s, k + 1);
    cta_gemm(gemm_args(keep, 2 * r2, r, b.R, 1, keep, Bn, 1, r, Cn, 1, keep), c.sm.e.u.gw.g);
    cta_sync();
    set_chi(c, s, k + 1, keep);
    if (ltid() == 0) b.bd[k + 1] = keep;
    cta_sync();
    cplx* t = C;
    C = Cn;
    Cn = t;
  }
  if (c.sm.fail) return;
  cta_copy(site_ptr(c, s, L - 1), C, (long long)b.bd[L - 1] * 2 * b.bd[L]);
  cta_sync();
  if (ltid() == 0) *s.oc = L - 1;
  cta_sync();
  normalize_state(c, s);  // truncate! ends with normalize!
}
