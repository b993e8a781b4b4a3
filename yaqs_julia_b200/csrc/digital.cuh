// digital.cuh — per-trajectory digital TJM program executed by one CTA.
//
// Restates run_digital_tjm (DigitalTJM.jl:363-450) with TEBD gate
// application (apply_local_gate_exact!, DigitalTJM.jl:251-305), SWAP chains
// for long-range gates (DigitalTJM.jl:314-330) and the local noise step
// after every 2-qubit gate (DigitalTJM.jl:405-420).
//
// The reference's noise step sweeps the whole chain (apply_dissipation walks
// the orthogonality centre from site L to 1, stochastic_process! contracts
// the full norm and normalize! re-canonicalises every site).  When every bond
// of the chain is "tight" (no bond exceeds twice either neighbour), the thin
// QR / LQ steps of those sweeps change no shape and are pure gauge moves:
// every dissipator and jump touches only the gate's sites, each is applied
// while the orthogonality centre sits on that site (as in the reference
// sweep), the norm equals the norm of the centre tensor and normalisation
// rescales it.  The device then performs the same operations at the gate's
// sites only, which is equivalent up to rounding; on a chain that is not
// tight, or with two-site dissipators that split, it runs the reference
// sweeps, so bond dimensions always match the reference's.
#pragma once
#include "tjm.cuh"

struct DevGate {
  int kind;  // 1 one-qubit, 2 two-qubit
  int a, b;  // sorted sites for 2-qubit gates (a < b)
  int wm;    // TDVP window: offset of its maps in DigParams::wm, -1 for TEBD
  cplx mat[16];
};

struct DigParams {
  const WMat* wm;  // per TDVP gate with window length n: heff1[n], heff2[n-1], envL[n], envR[n]
  const DevGate* gates;
  const int* layer_off;   // [n_layers + 1] into gates
  const int* sample_col;  // [n_layers] measurement column after the layer, -1 for none
  int n_layers;
  int sample_at_start;
  int any_sample;
};

static __device__ __constant__ cplx c_swap[16] = {{1, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {1, 0}, {0, 0},
                                           {0, 0}, {1, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {1, 0}};

// apply_local_gate_exact! on sites (s1, s1+1).
static __device__ void tebd_apply(Ctx& c, const DState& s, const cplx* op, int s1) {
  ProfScope prof_scope_(PF_SWEEP);
  shift_oc(c, s, s1);
  if (c.sm.fail) return;
  cplx* th = c.ws + c.P.lay.th;
  const int l = s.chi[s1], r = s.chi[s1 + 2];
  const int k = s.chi[s1 + 1];
  merge(c, s, s1, th);
  apply_local(th, l, 4, r, op);
  split(c, s, s1, th, l, r, 2, false);
  cta_sync();
  if (ltid() == 0) {
    *s.oc = s1 + 1;
    // nominal work: theta merge GEMM, 4x4 gate, SVD counted as 4 m n min(m, n) complex MACs
    const double m = 2.0 * l, n = 2.0 * r;
    *c.fl += 8.0 * (m * n * k + 4.0 * m * n + 4.0 * m * n * fmin(m, n));
  }
  cta_sync();
}

// apply_window! with method :TEBD (DigitalTJM.jl:307-334).
static __device__ void apply_window_tebd(Ctx& c, const DState& s, const DevGate& g) {
  if (g.b > g.a + 1) {
    for (int k = g.b - 1; k >= g.a + 1 && !c.sm.fail; --k) tebd_apply(c, s, c_swap, k);
    if (!c.sm.fail) tebd_apply(c, s, g.mat, g.a);
    for (int k = g.a + 1; k <= g.b - 1 && !c.sm.fail; ++k) tebd_apply(c, s, c_swap, k);
  } else {
    tebd_apply(c, s, g.mat, g.a);
  }
}

// apply_window! with method :TDVP (DigitalTJM.jl:335-358): the window
// a..b evolves under the product MPO coeff g1 (x) 1 ... 1 (x) g2
// (construct_window_mpo, DigitalTJM.jl:192-236) by one forward circuit 2-site
// sweep (_tdvp_sweep_circuit_2site!, Algorithms.jl:606-627): each pair by +1
// with the right site back-evolved by -1 (:631-672), the last pair by +1
// split to the right (:762-800); the centre ends on b.
static __device__ void apply_window_tdvp(Ctx& c, const DState& s, const DevGate& g, const WMat* wm) {
  const int s1 = g.a, s2 = g.b, n = s2 - s1 + 1;
  const WMat* h1 = wm;
  const WMat* h2 = wm + n;
  const WMat* eL = wm + 2 * n - 1;
  const WMat* eR = wm + 3 * n - 1;
  cplx* th = c.ws + c.P.lay.th;
  shift_oc(c, s, s1);
  if (c.sm.fail) return;
  identity_env(c, envL(c, s1), s.chi[s1], 1);
  identity_env(c, envR(c, s2 + 1), s.chi[s2 + 1], 1);
  for (int j = n - 1; j >= 1; --j) update_right_w(c, s, s1 + j, eR[j]);
  for (int j = 0; j + 2 < n && !c.sm.fail; ++j) {
    const int i = s1 + j, l = s.chi[i], r = s.chi[i + 2];
    merge(c, s, i, th);
    evolve(c, th, l, 4, r, i, i + 2, h2[j], 1.0);
    split(c, s, i, th, l, r, 0, false);
    if (c.sm.fail) return;
    update_left_w(c, s, i, eL[j]);
    evolve(c, site_ptr(c, s, i + 1), s.chi[i + 1], 2, r, i + 1, i + 2, h1[j + 1], -1.0);
  }
  if (c.sm.fail) return;
  const int i = s2 - 1, l = s.chi[i], r = s.chi[i + 2];
  merge(c, s, i, th);
  evolve(c, th, l, 4, r, i, i + 2, h2[n - 2], 1.0);
  split(c, s, i, th, l, r, 0, false);  // the centre moves to s2
}

// Local dissipation (dt = 1) and jump step after a 2-qubit gate on (s1, s2),
// s1 < s2 (DigitalTJM.jl:405-420).  When the chain is tight and no
// dissipator needs a two-site split, every operation of the reference sweeps
// away from the gate's sites is a gauge move, and only the gate's sites are
// visited; otherwise the reference sweeps run as they are.
static __device__ void digital_noise(Ctx& c, const DState& s, int s1, int s2) {
  ProfScope prof_scope_(PF_STOCH);
  const DevParams& P = c.P;
  int nloc = 0;
  bool all_zero = true, split_diss = false, scalar_only = true, has_lr = false;
  double fdiss = 1.0;
  for (int k = 0; k < P.nprocs; ++k) {
    const DevProc& pr = P.procs[k];
    if (!proc_on(pr, s1, s2)) continue;
    ++nloc;
    if (pr.gamma != 0.0) all_zero = false;
    if (pr.nsites == 2 && !pr.pauli_name) split_diss = true;
    if (pr.nsites != 1 || !pr.pauli_name || !pr.pauli_proc || !pr.unitary) scalar_only = false;
    if (pr.lr) has_lr = true;
    fdiss *= exp(-0.5 * pr.drate);
  }
  if (!P.noise_present || nloc == 0) {
    finish_normalize(c, s);
    return;
  }
  const bool tight = chain_tight(c, s);
  if ((split_diss && !all_zero) || !tight || has_lr) {  // long-range jumps need the full sweeps
    apply_dissipation(c, s, true, 1.0, s1, s2);
    if (c.sm.fail) return;
    stochastic_process(c, s, 1.0, s1, s2);
    return;
  }
  if (scalar_only) {
    // Pauli processes on single sites: every dissipator is a scalar, every
    // candidate weight is gamma times the state norm, and a unitary jump on
    // any site keeps the gauge, so nothing needs the centre moved.
    const int oc = *s.oc;
    cplx* A = site_ptr(c, s, oc);
    const long long n = (long long)s.chi[oc] * 2 * s.chi[oc + 1];
    if (!all_zero) {
      cta_scale(A, n, fdiss);
      cta_sync();
    }
    const double nrm = cta_norm2(A, n, c.sm.e.r);
    const double u1 = draw_uniform(c);
    if (u1 >= 1.0 - nrm) {
      normalize_center(c, s);
      return;
    }
    double total = 0.0;
    for (int k = 0; k < P.nprocs; ++k)
      if (proc_on(P.procs[k], s1, s2)) total += P.procs[k].gamma * nrm;
    if (total == 0.0) {
      normalize_center(c, s);
      return;
    }
    const double r = draw_uniform(c);
    double acc = 0.0;
    int chosen = -1, first = -1;
    const int sites[2] = {s1, s2};
    for (int si = 0; si < 2 && chosen < 0; ++si)
      for (int k = 0; k < P.nprocs && chosen < 0; ++k) {
        const DevProc& pr = P.procs[k];
        if (!proc_on(pr, s1, s2) || pr.s0 != sites[si]) continue;
        if (first < 0) first = k;
        acc += pr.gamma * nrm / total;
        if (r <= acc) chosen = k;
      }
    if (chosen < 0) chosen = first;  // rounding left the cumulative sum below r: the first candidate
    const DevProc& pr = P.procs[chosen];
    apply_local(site_ptr(c, s, pr.s0), s.chi[pr.s0], 2, s.chi[pr.s0 + 1], pr.mat);
    if (ltid() == 0) c.cnt[3] += 1;
    normalize_center(c, s);
    return;
  }
  cplx* th = c.ws + c.P.lay.th;
  // apply_dissipation: the reference sweep reaches s2 before s1
  if (!all_zero) {
    const int sites[2] = {s2, s1};
    for (int si = 0; si < 2 && !c.sm.fail; ++si) {
      const int i = sites[si];
      shift_oc(c, s, i);
      for (int k = 0; k < P.nprocs; ++k) {
        const DevProc& pr = P.procs[k];
        if (!proc_on(pr, s1, s2) || pr.nsites != 1 || pr.s0 != i) continue;
        cplx* A = site_ptr(c, s, i);
        if (pr.pauli_name) {
          cta_scale(A, (long long)s.chi[i] * 2 * s.chi[i + 1], exp(-0.5 * pr.gamma));
          cta_sync();
        } else {
          apply_local(A, s.chi[i], 2, s.chi[i + 1], pr.diss_full);
        }
      }
      if (si == 0) {  // 2-site Pauli processes on (s1, s2) scale site s2
        for (int k = 0; k < P.nprocs; ++k) {
          const DevProc& pr = P.procs[k];
          if (!proc_on(pr, s1, s2) || pr.nsites != 2 || pr.s1 != i) continue;
          cta_scale(site_ptr(c, s, i), (long long)s.chi[i] * 2 * s.chi[i + 1], exp(-0.5 * pr.drate));
          cta_sync();
        }
      }
    }
  }
  if (c.sm.fail) return;
  // stochastic_process!: the norm is the norm of the centre tensor
  const int oc = *s.oc;
  const double nrm = cta_norm2(site_ptr(c, s, oc), (long long)s.chi[oc] * 2 * s.chi[oc + 1], c.sm.e.r);
  const double dp = 1.0 - nrm;
  const double u1 = draw_uniform(c);
  if (u1 >= dp) {
    normalize_center(c, s);
    return;
  }
  double* cand = reinterpret_cast<double*>(c.ws + c.P.lay.dbl) + SVD_MAX_COLS;
  int* candp = c.wsi + c.P.lay.i_cand;
  int nc = 0;
  const int sites[2] = {s1, s2};
  for (int si = 0; si < 2 && !c.sm.fail; ++si) {
    const int site = sites[si];
    shift_oc(c, s, site);
    for (int k = 0; k < P.nprocs; ++k) {
      const DevProc& pr = P.procs[k];
      if (!proc_on(pr, s1, s2) || pr.nsites != 1 || pr.s0 != site) continue;
      double nr = local_norm2(c, site_ptr(c, s, site), s.chi[site], 2, s.chi[site + 1], pr.pauli_proc ? nullptr : pr.mat);
      if (ltid() == 0) {
        cand[nc] = pr.gamma * nr;
        candp[nc] = k;
      }
      ++nc;
    }
    if (site < P.L - 1) {
      for (int k = 0; k < P.nprocs; ++k) {
        const DevProc& pr = P.procs[k];
        if (!proc_on(pr, s1, s2) || pr.nsites != 2 || pr.s0 != site) continue;
        double nr;
        if (pr.pauli_proc) {
          nr = local_norm2(c, site_ptr(c, s, site), s.chi[site], 2, s.chi[site + 1], nullptr);
        } else {
          merge(c, s, site, th);
          nr = local_norm2(c, th, s.chi[site], 4, s.chi[site + 2], pr.mat);
        }
        if (ltid() == 0) {
          cand[nc] = pr.gamma * nr;
          candp[nc] = k;
        }
        ++nc;
      }
    }
  }
  cta_sync();
  double total = 0.0;
  for (int e = 0; e < nc; ++e) total += cand[e];
  if (total == 0.0) {
    normalize_center(c, s);
    return;
  }
  const double r = draw_uniform(c);
  double acc = 0.0;
  int chosen = 0;
  for (int e = 0; e < nc; ++e) {
    acc += cand[e] / total;
    if (r <= acc) {
      chosen = e;
      break;
    }
  }
  const DevProc& pr = P.procs[candp[chosen]];
  cta_sync();
  shift_oc(c, s, pr.s0);
  if (pr.nsites == 1) {
    apply_local(site_ptr(c, s, pr.s0), s.chi[pr.s0], 2, s.chi[pr.s0 + 1], pr.mat);
  } else {
    const int l = s.chi[pr.s0], rr = s.chi[pr.s0 + 2];
    merge(c, s, pr.s0, th);
    apply_local(th, l, 4, rr, pr.mat);
    split(c, s, pr.s0, th, l, rr, 1, false);
  }
  if (ltid() == 0) c.cnt[3] += 1;
  finish_normalize(c, s);
}

// Launch 0: initial state, normalisation and the start sample; launch l >= 1:
// layer l-1 (its 1-qubit gates first, then each 2-qubit gate followed by the
// noise step) and the sample after it.
static __device__ void run_digital_step(Ctx& c, const DigParams& D, int launch) {
  ProfScope prof_scope_(PF_STEP);
  const DevParams& P = c.P;
  const int L = P.L;
  DState st{P.phi + (long long)c.traj * P.mps_size, P.phi_chi + (long long)c.traj * (L + 1), P.phi_oc + c.traj};
  if (launch == 0) {
    cta_copy(st.a, P.psi0, P.mps_size);
    for (int b = ltid(); b <= L; b += NT) st.chi[b] = P.chi0[b];
    if (ltid() == 0) *st.oc = 0;
    cta_sync();
    normalize_state(c, st);  // Simulator.jl:128
    if (D.sample_at_start) evaluate(c, st, 0);
    if (D.n_layers == 0 && !D.any_sample && P.nobs > 0) evaluate(c, st, 0);
    return;
  }
  const int l = launch - 1;
  for (int g = D.layer_off[l]; g < D.layer_off[l + 1]; ++g) {
    const DevGate& G = D.gates[g];
    if (G.kind == 1) apply_local(site_ptr(c, st, G.a), st.chi[G.a], 2, st.chi[G.a + 1], G.mat);
  }
  for (int g = D.layer_off[l]; g < D.layer_off[l + 1] && !c.sm.fail; ++g) {
    const DevGate& G = D.gates[g];
    if (G.kind != 2) continue;
    if (G.wm >= 0)
      apply_window_tdvp(c, st, G, D.wm + G.wm);
    else
      apply_window_tebd(c, st, G);
    if (c.sm.fail) return;
    digital_noise(c, st, G.a, G.b);
    if (c.sm.fail) return;
    if (ltid() == 0) c.cnt[6] += 1;
  }
  if (c.sm.fail) return;
  if (D.sample_col[l] >= 0) evaluate(c, st, D.sample_col[l]);
  if (l == D.n_layers - 1 && !D.any_sample && P.nobs > 0) evaluate(c, st, 0);
}
