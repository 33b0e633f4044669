// pmc_replay.cu -- one device thread replays mc_coag in the reference's order.
//
// Compiled with -fmad=false: every multiply and add is rounded separately,
// as in the reference's gfortran build, so that particle volumes (sums of
// the same terms in the same order) match the CPU restatement bit for bit.
// Functions follow src/coagulation.F90 and the modules it calls; each names
// the routine it restates.
#include "pmc_replay.cuh"

#include "pmc_particle.cuh"
#include "pmc_physics.cuh"

namespace pmc {
namespace {

struct Src {
  const double* u;
  long long n, pos;
  bool ok;
  __device__ double next() {
    if (pos >= n) {
      ok = false;
      return 0.5;
    }
    return u[pos++];
  }
};

struct Tp {  // a particle outside the array (accumulator, copy)
  double vol[kMaxSpec];
  PMeta m;
};

struct Seq {
  const PopDev* P;
  ReplayDev R;
  Src g;
  int n;  // particles
  int status;
  int nb;
  const GridDev* G;
  long long samp, coag;

  __device__ bool fail(int code) {
    if (!status) status = code;
    return false;
  }
  __device__ bool rng_ok() { return g.ok ? true : fail(kErrRng); }

  // ---- particle slots (aero_particle_array, aero_particle_array.F90:158-198)
  __device__ double vtot(int i) { return P->vtot[i - 1]; }
  __device__ double radius(int i) { return vol2rad(P->benv.frac, P->vtot[i - 1]); }
  __device__ void load(int i, Tp& t) {
    for (int s = 0; s < P->n_spec; s++) t.vol[s] = P->vol[vol_at(*P, i - 1, s)];
    load_meta(*P, i - 1, t.m);
  }
  __device__ void copy_slot(int dst, int src) {
    Tp t;
    load(src, t);
    store_particle(*P, dst - 1, t.vol, t.m);
  }
  __device__ bool array_remove(int i) {
    if (i < 1 || i > n) return fail(kErrAssert);
    if (i < n) copy_slot(i, n);
    P->alive[n - 1] = 0;
    P->changed[n - 1] = 1;
    n--;
    return true;
  }
  __device__ bool array_add(const Tp& t) {
    if (n >= P->cap) return fail(kErrCapacity);
    n++;
    store_particle(*P, n - 1, t.vol, t.m);
    return true;
  }

  // ---- integer_rmap2 (integer_rmap2.F90:107-243), values 1-based
  __device__ int* cell(RMapDev& m, int j1, int j2) {
    return m.inv + (size_t)((j1 - 1) + m.n_r1 * (j2 - 1)) * m.cap;
  }
  __device__ int& cell_n(RMapDev& m, int j1, int j2) { return m.inv_n[(j1 - 1) + m.n_r1 * (j2 - 1)]; }
  __device__ bool cell_push(RMapDev& m, int j1, int j2, int x) {
    int& c = cell_n(m, j1, j2);
    if (c >= m.cap) return fail(kErrCapacity);
    cell(m, j1, j2)[c] = x;
    c++;
    return true;
  }
  // integer_varray_remove_entry (integer_varray.F90:151-171) on a cell
  __device__ bool cell_remove_entry(RMapDev& m, int j1, int j2, int idx) {
    int& c = cell_n(m, j1, j2);
    if (idx < 1 || idx > c) return fail(kErrAssert);
    int* e = cell(m, j1, j2);
    if (idx < c) e[idx - 1] = e[c - 1];
    e[c - 1] = 0;
    c--;
    return true;
  }
  __device__ void rmap_zero(RMapDev& m) {
    *m.n = 0;
    for (int k = 0; k < m.n_r1 * m.n_r2; k++) m.inv_n[k] = 0;
  }
  __device__ bool rmap_append(RMapDev& m, int j1, int j2) {
    if (j1 < 1 || j1 > m.n_r1 || j2 < 1 || j2 > m.n_r2) return fail(kErrAssert);
    int d = *m.n;
    if (d >= m.cap) return fail(kErrCapacity);
    m.fwd1[d] = j1;
    m.fwd2[d] = j2;
    *m.n = d + 1;
    if (!cell_push(m, j1, j2, d + 1)) return false;
    m.index[d] = cell_n(m, j1, j2);
    return true;
  }
  // integer_rmap2_change, with the reference's early return on an unchanged
  // first range (integer_rmap2.F90:160)
  __device__ bool rmap_change(RMapDev& m, int i, int j1, int j2) {
    if (i < 1 || i > *m.n || j1 < 1 || j1 > m.n_r1 || j2 < 1 || j2 > m.n_r2) return fail(kErrAssert);
    int o1 = m.fwd1[i - 1], o2 = m.fwd2[i - 1];
    if (o1 == j1) return true;
    int idx_old = m.index[i - 1];
    if (!cell_remove_entry(m, o1, o2, idx_old)) return false;
    if (idx_old <= cell_n(m, o1, o2)) {
      int shifted = cell(m, o1, o2)[idx_old - 1];
      m.index[shifted - 1] = idx_old;
    }
    m.fwd1[i - 1] = j1;
    m.fwd2[i - 1] = j2;
    if (!cell_push(m, j1, j2, i)) return false;
    m.index[i - 1] = cell_n(m, j1, j2);
    return true;
  }
  // integer_rmap2_remove (integer_rmap2.F90:190-243)
  __device__ bool rmap_remove(RMapDev& m, int i) {
    int nd = *m.n;
    if (i < 1 || i > nd) return fail(kErrAssert);
    int o1 = m.fwd1[i - 1], o2 = m.fwd2[i - 1], idx_old = m.index[i - 1];
    int shifted = nd;
    if (shifted != i) {
      int f1 = m.fwd1[shifted - 1], f2 = m.fwd2[shifted - 1], fi = m.index[shifted - 1];
      cell(m, f1, f2)[fi - 1] = i;
    }
    // varray_remove_entry on the three forward arrays
    if (i < nd) {
      m.fwd1[i - 1] = m.fwd1[nd - 1];
      m.fwd2[i - 1] = m.fwd2[nd - 1];
      m.index[i - 1] = m.index[nd - 1];
    }
    m.fwd1[nd - 1] = m.fwd2[nd - 1] = m.index[nd - 1] = 0;
    *m.n = nd - 1;
    int idx_fix = cell_n(m, o1, o2);
    int dom_fix = cell(m, o1, o2)[idx_fix - 1];
    if (!cell_remove_entry(m, o1, o2, idx_old)) return false;
    if (idx_fix != idx_old) m.index[dom_fix - 1] = idx_old;
    return true;
  }

  __device__ int in_bin(double r) { return bin_find(nb, G->log_lo, G->log_hi, r); }

  // aero_sorted_sort_particles (aero_sorted.F90:185-209)
  __device__ bool sort_particles() {
    rmap_zero(R.size_class);
    rmap_zero(R.group_class);
    for (int i = 1; i <= n; i++) {
      int b = in_bin(radius(i));
      if (!rmap_append(R.size_class, b, P->cls[i - 1])) return false;
      if (!rmap_append(R.group_class, P->grp[i - 1], P->cls[i - 1])) return false;
    }
    return true;
  }

  // aero_state_remove_particle with a valid sort (aero_sorted.F90:455-470)
  __device__ bool state_remove(int i) {
    if (!array_remove(i)) return false;
    if (!rmap_remove(R.size_class, i)) return false;
    return rmap_remove(R.group_class, i);
  }
  // aero_state_add_particle / aero_sorted_add_particle (aero_sorted.F90:397-449);
  // a particle off the grid is an error here (the reference remakes the grid
  // when allowed, which only the host can do)
  __device__ bool state_add(const Tp& t) {
    double vt = 0.0;
    for (int s = 0; s < P->n_spec; s++) vt = vt + t.vol[s];
    int b = in_bin(vol2rad(P->benv.frac, vt));
    if (t.m.grp < 1 || t.m.grp > P->n_group || t.m.cls < 1 || t.m.cls > P->n_class) return fail(kErrAssert);
    if (!array_add(t)) return false;
    if (b < 1 || b > nb) return fail(kErrOutOfGrid);
    if (!rmap_append(R.size_class, b, t.m.cls)) return false;
    return rmap_append(R.group_class, t.m.grp, t.m.cls);
  }

  __device__ long long new_id() {
    long long id = *R.next_id;
    *R.next_id = id + 1;
    return id;
  }

  // aero_state_dup_particle with random_weight_group (aero_state.F90:488-539)
  __device__ bool state_dup(int i, double n_mean) {
    int nc = prob_round(g, n_mean);
    if (!rng_ok()) return false;
    if (nc == 0) {
      log_removal(*P, P->id[i - 1], kInfoWeight, 0);
      return state_remove(i);
    }
    for (int d = 1; d <= nc - 1; d++) {
      Tp c;
      load(i, c);
      c.m.id = new_id();
      int grp = rand_group(g, P->w, P->cls[i - 1] - 1, radius(i));
      if (!rng_ok()) return false;
      if (grp == 0) return fail(kErrTimeout);
      c.m.grp = grp;
      if (!state_add(c)) return false;
    }
    return true;
  }

  __device__ int cn(int b, int c) { return cell_n(R.size_class, b, c); }
  __device__ int ce(int b, int c, int k) { return cell(R.size_class, b, c)[k - 1]; }

  // num_conc_weighted_kernel on two volume vectors (coag_kernel.F90:175-209)
  __device__ bool weighted_kernel(const double* va, const double* vb, int ci, int cj, int cij,
                                  double* k) {
    double v1 = 0.0, v2 = 0.0, m1 = 0.0, m2 = 0.0;
    for (int s = 0; s < P->n_spec; s++) {
      v1 = v1 + va[s];
      v2 = v2 + vb[s];
    }
    double kk = 0.0;
    bool ok = true;
    switch (P->kernel_type) {
      case kKernelSedi:
        kk = sedi_kernel(P->benv, v1, v2, &ok);
        if (kk < 0.0) return fail(kErrAssert);
        break;
      case kKernelAdditive: kk = P->coeff * (v1 + v2); break;
      case kKernelConstant: kk = kBeta0; break;
      case kKernelBrown:
        for (int s = 0; s < P->n_spec; s++) {
          m1 = m1 + va[s] * P->density[s];
          m2 = m2 + vb[s] * P->density[s];
        }
        kk = brown_kernel(P->benv, v1, m1 / v1, v2, m2 / v2, &ok);
        break;
      case kKernelBrownFree:
        for (int s = 0; s < P->n_spec; s++) {
          m1 = m1 + va[s] * P->density[s];
          m2 = m2 + vb[s] * P->density[s];
        }
        kk = brown_free_kernel(P->benv, v1, m1 / v1, v2, m2 / v2);
        break;
      case kKernelBrownCont: kk = brown_cont_kernel(P->benv, v1, v2); break;
      default: kk = 0.0;
    }
    if (!ok) return fail(kErrAssert);  // the fractal Newton loop did not converge
    const Fractal& F = P->benv.frac;
    double ri = vol2rad(F, v1), rj = vol2rad(F, v2);
    *k = kk * num_conc_factor(P->w, F, ri, rj, ci - 1, cj - 1, cij - 1);
    return true;
  }
  __device__ void slot_vol(int i, double* v) {
    for (int s = 0; s < P->n_spec; s++) v[s] = P->vol[vol_at(*P, i - 1, s)];
  }

  // coagulate_weighting + coagulate (coagulation.F90:810-985)
  __device__ bool coagulate(int p1, int p2, int c1, int c2, int cc) {
    if (P->id[p1 - 1] == P->id[p2 - 1]) return fail(kErrAssert);
    double r1 = radius(p1), r2 = radius(p2);
    double rc = vol2rad(P->benv.frac, rad2vol(P->benv.frac, r1) + rad2vol(P->benv.frac, r2));
    double nc1 = num_conc_at_radius<double>(P->w, c1 - 1, r1);
    double nc2 = num_conc_at_radius<double>(P->w, c2 - 1, r2);
    double ncc = num_conc_at_radius<double>(P->w, cc - 1, rc);
    int new_group = rand_group(g, P->w, cc - 1, rc);
    if (!rng_ok()) return false;
    if (new_group == 0) return fail(kErrTimeout);
    double mn = nc1;
    if (nc2 < mn) mn = nc2;
    if (ncc < mn) mn = ncc;
    bool rm1 = g.next() < mn / nc1;
    bool rm2 = g.next() < mn / nc2;
    bool cn_ = g.next() < mn / ncc;
    if (!rng_ok()) return false;
    bool l1, l2;
    if (cn_) {
      l1 = l2 = false;
      if (rm1 && rm2) {
        if (vtot(p1) > vtot(p2)) l2 = true;
        else l1 = true;
      }
    } else {
      l1 = rm1;
      l2 = rm2;
    }
    Tp ptc;
    if (cn_) {
      Tp a, b;
      load(p1, a);
      load(p2, b);
      double ia = 0.0, ib = 0.0;
      if (P->i_water > 0) {
        ia = a.vol[P->i_water - 1];
        ib = b.vol[P->i_water - 1];
      }
      coag_meta(g, a.m, ia, b.m, ib, ptc.m);
      if (!rng_ok()) return false;
      for (int s = 0; s < P->n_spec; s++) ptc.vol[s] = a.vol[s] + b.vol[s];
      ptc.m.grp = new_group;
      ptc.m.cls = cc;
      if (rm1 && !l1) ptc.m.id = a.m.id;
      else if (rm2 && !l2) ptc.m.id = b.m.id;
      else ptc.m.id = new_id();
    }
    // aero_info of each removal whose ID is lost, in the order of removal
    const long long id1 = P->id[p1 - 1], id2 = P->id[p2 - 1], other = cn_ ? ptc.m.id : 0;
    if (p2 > p1) {
      if (rm2 && l2) log_removal(*P, id2, kInfoCoag, other);
      if (rm2 && !state_remove(p2)) return false;
      if (rm1 && l1) log_removal(*P, id1, kInfoCoag, other);
      if (rm1 && !state_remove(p1)) return false;
    } else {
      if (rm1 && l1) log_removal(*P, id1, kInfoCoag, other);
      if (rm1 && !state_remove(p1)) return false;
      if (rm2 && l2) log_removal(*P, id2, kInfoCoag, other);
      if (rm2 && !state_remove(p2)) return false;
    }
    if (cn_) return state_add(ptc);
    return true;
  }

  // maybe_coag_pair + find_rand_pair (coagulation.F90:712-803)
  __device__ bool maybe_coag_pair(int b1, int b2, int c1, int c2, int cc, double af, bool* did) {
    int n1 = cn(b1, c1), n2 = cn(b2, c2);
    if (n1 < 1) return fail(kErrAssert);
    int i1 = rand_int(g, n1), i2;
    if (b1 == b2 && c1 == c2) {
      if (n2 < 2) return fail(kErrAssert);
      i2 = rand_int(g, n2 - 1);
      if (i2 == i1) i2 = n2;
    } else {
      if (n2 < 1) return fail(kErrAssert);
      i2 = rand_int(g, n2);
    }
    if (!rng_ok()) return false;
    int p1 = ce(b1, c1, i1), p2 = ce(b2, c2, i2);
    double v1[kMaxSpec], v2[kMaxSpec], k;
    slot_vol(p1, v1);
    slot_vol(p2, v2);
    if (!weighted_kernel(v1, v2, c1, c2, cc, &k)) return false;
    double p = k * af;
    *did = false;
    if (g.next() < p) {
      if (!rng_ok()) return false;
      if (!coagulate(p1, p2, c1, c2, cc)) return false;
      *did = true;
    }
    return rng_ok();
  }

  // per_set_coag + compute_n_samp (coagulation.F90:587-702)
  __device__ bool per_set(double k_max, int b1, int b2, int c1, int c2, int cc) {
    int n1 = cn(b1, c1), n2 = cn(b2, c2);
    bool same = b1 == b2 && c1 == c2;
    double n_possible = same ? (double)n1 * ((double)n2 - 1.0) / 2.0 : (double)n1 * (double)n2;
    double r_samp = k_max * P->del_t;
    double mean = r_samp * n_possible;
    int ns = rand_poisson(g, mean);
    if (!rng_ok()) return false;
    if (ns < 0) return fail(kErrTimeout);
    double af = 1.0 / k_max;
    samp += ns;
    for (int s = 1; s <= ns; s++) {
      n1 = cn(b1, c1);
      n2 = cn(b2, c2);
      if ((n1 < 2 && same) || n1 < 1 || n2 < 1) break;
      bool did;
      if (!maybe_coag_pair(b1, b2, c1, c2, cc, af, &did)) return false;
      if (did) coag++;
    }
    return true;
  }

  // sample_source_particle (coagulation.F90:333-517)
  __device__ bool sample_source(int bs, int cs, const Tp& target, double nspt, double af,
                                int* n_samp_out, int* n_coag_out, Tp& src) {
    int ns = P->n_spec;
    *n_samp_out = 0;
    *n_coag_out = 0;
    if (cn(bs, cs) == 0) return true;
    double vt = 0.0;
    for (int s = 0; s < ns; s++) vt = vt + target.vol[s];
    int ct = target.m.cls;
    double nc_target = num_conc_at_radius<double>(P->w, ct - 1, vol2rad(P->benv.frac, vt));
    double nc_src_min = num_conc_at_radius<double>(P->w, cs - 1, G->edges[bs - 1]);
    double prm_max = nc_target / nc_src_min;
    if (!(prm_max <= 1.0)) return fail(kErrAssert);
    int n_remove = rand_poisson(g, prm_max * nspt);
    int n_extra = rand_poisson(g, (1.0 - prm_max) * nspt);
    if (!rng_ok()) return false;
    if (n_remove < 0 || n_extra < 0) return fail(kErrTimeout);
    int n_total = n_remove + n_extra;
    int n_avg = 0, n_samp = 0;
    double pc_tot = 0.0;
    double vol_sq[kMaxSpec], vol_cv[kMaxSpec];
    for (int s = 0; s < ns; s++) {
      vol_sq[s] = 0.0;
      vol_cv[s] = 0.0;
      src.vol[s] = 0.0;
    }
    zero_meta(src.m);
    for (int i_samp = 1; i_samp <= n_total; i_samp++) {
      if (cn(bs, cs) == 0) break;
      if (n_samp > n_remove && n_avg >= 2) {
        double cv_max = 0.0;
        bool found = false;
        for (int s = 0; s < ns; s++) {
          double mean = src.vol[s] / (double)n_avg;
          if (mean > 0.0) vol_cv[s] = sqrt(vol_sq[s] / (double)n_avg - mean * mean) / mean;
        }
        for (int s = 0; s < ns; s++) {
          if (isnan(vol_cv[s])) continue;
          if (!found || vol_cv[s] > cv_max) cv_max = vol_cv[s];
          found = true;
        }
        if (!found) cv_max = __longlong_as_double(0x7ff8000000000000LL);
        double conf = cv_max / sqrt((double)n_avg) * student_t_95(n_avg);
        if (conf < 0.1) break;
      }
      n_samp++;
      int ie = rand_int(g, cn(bs, cs));
      if (!rng_ok()) return false;
      int ip = ce(bs, cs, ie);
      double vi[kMaxSpec], k;
      slot_vol(ip, vi);
      if (!weighted_kernel(vi, target.vol, cs, ct, ct, &k)) return false;
      double pc = k * af;
      pc_tot = pc_tot + pc;
      if (g.next() < pc) {
        n_avg++;
        PMeta im;
        load_meta(*P, ip - 1, im);
        double ia = 0.0, ib = 0.0;
        if (P->i_water > 0) {
          ia = src.vol[P->i_water - 1];
          ib = vi[P->i_water - 1];
        }
        coag_meta(g, src.m, ia, im, ib, src.m);
        for (int s = 0; s < ns; s++) src.vol[s] = src.vol[s] + vi[s];
        for (int s = 0; s < ns; s++) vol_sq[s] = vol_sq[s] + vi[s] * vi[s];
        if (i_samp <= n_remove) {
          double nc_i = num_conc_at_radius<double>(P->w, P->cls[ip - 1] - 1, radius(ip));
          double pri = nc_target / nc_i;
          if (g.next() < pri / prm_max) {
            if (!rng_ok()) return false;
            log_removal(*P, P->id[ip - 1], kInfoCoag, target.m.id);
            if (!state_remove(ip)) return false;
          }
        }
      }
      if (!rng_ok()) return false;
    }
    *n_samp_out = n_samp;
    if (n_avg == 0) return true;
    double pc_mean = pc_tot / (double)n_samp;
    int n_coag = rand_binomial(g, n_total, pc_mean);
    if (!rng_ok()) return false;
    *n_coag_out = n_coag;
    for (int s = 0; s < ns; s++) src.vol[s] = src.vol[s] * ((double)n_coag / (double)n_avg);
    src.m.nprim = prob_round(g, (double)src.m.nprim * ((double)n_coag / (double)n_avg));
    if (!rng_ok()) return false;
    int n_comp = src.m.ncomp;
    int n_new = src.m.nprim < kMaxComponent ? src.m.nprim : kMaxComponent;
    int sample[kMaxComponent];
    if (n_new < n_comp) {
      PMeta m = src.m;
      sample_wo_replacement(g, n_new, n_comp, sample);
      for (int i = 0; i < n_new; i++) {
        m.csrc[i] = src.m.csrc[sample[i] - 1];
        m.ctime[i] = src.m.ctime[sample[i] - 1];
      }
      m.ncomp = n_new;
      src.m = m;
    } else if (n_comp < kMaxComponent) {
      if (n_comp == 0 && n_new > 0) return fail(kErrAssert);
      PMeta m = src.m;
      int i_comp = 1;
      while (i_comp <= n_new) {
        if (i_comp + n_comp <= n_new) {
          for (int i = 1; i <= n_comp; i++) {
            m.csrc[i_comp + i - 2] = src.m.csrc[i - 1];
            m.ctime[i_comp + i - 2] = src.m.ctime[i - 1];
          }
          i_comp += n_comp;
        } else {
          int size = n_new - i_comp + 1;
          sample_wo_replacement(g, size, n_comp, sample);
          for (int i = 1; i <= size; i++) {
            m.csrc[i_comp + i - 2] = src.m.csrc[sample[i - 1] - 1];
            m.ctime[i_comp + i - 2] = src.m.ctime[sample[i - 1] - 1];
          }
          i_comp = n_new + 1;
        }
      }
      m.ncomp = n_new;
      src.m = m;
    }
    if (src.m.nprim < src.m.ncomp) return fail(kErrAssert);
    return rng_ok();
  }

  // coag_target_with_source (coagulation.F90:522-582)
  __device__ bool target_with_source(int bt, int ct, int entry, const Tp& src, int cc) {
    int tp = ce(bt, ct, entry);
    long long tid = P->id[tp - 1];
    double old_nc = num_conc_at_radius<double>(P->w, P->cls[tp - 1] - 1, radius(tp));
    Tp t;
    load(tp, t);
    double it = 0.0, is = 0.0;
    if (P->i_water > 0) {
      it = t.vol[P->i_water - 1];
      is = src.vol[P->i_water - 1];
    }
    PMeta nm;
    coag_meta(g, t.m, it, src.m, is, nm);
    if (!rng_ok()) return false;
    for (int s = 0; s < P->n_spec; s++) t.vol[s] = t.vol[s] + src.vol[s];
    nm.id = tid;
    t.m = nm;
    double vt = 0.0;
    for (int s = 0; s < P->n_spec; s++) vt = vt + t.vol[s];
    int grp = rand_group(g, P->w, cc - 1, vol2rad(P->benv.frac, vt));
    if (!rng_ok()) return false;
    if (grp == 0) return fail(kErrTimeout);
    t.m.grp = grp;
    t.m.cls = cc;
    store_particle(*P, tp - 1, t.vol, t.m);
    int nbn = in_bin(radius(tp));
    if (nbn < 1 || nbn > nb) return fail(kErrOutOfGrid);
    if (!rmap_change(R.size_class, tp, nbn, cc)) return false;
    if (!rmap_change(R.group_class, tp, grp, cc)) return false;
    double new_nc = num_conc_at_radius<double>(P->w, cc - 1, radius(tp));
    if (!state_dup(tp, old_nc / new_nc)) return false;
    if (P->id[tp - 1] != tid) return fail(kErrAssert);
    return true;
  }

  // try_per_particle_coag (coagulation.F90:150-241); *done = path taken
  __device__ bool try_per_particle(double k_max, int b1, int b2, int c1, int c2, int cc, bool* done) {
    *done = false;
    bool inc, dec;
    weight_monotonicity(P->w, &inc, &dec);
    if (!dec) return true;
    if (!(inc || dec)) return fail(kErrAssert);
    double a, b;
    a = num_conc_at_radius<double>(P->w, c1 - 1, G->edges[b1 - 1]);
    b = num_conc_at_radius<double>(P->w, c1 - 1, G->edges[b1]);
    double n1min = a < b ? a : b, n1max = a > b ? a : b;
    a = num_conc_at_radius<double>(P->w, c2 - 1, G->edges[b2 - 1]);
    b = num_conc_at_radius<double>(P->w, c2 - 1, G->edges[b2]);
    double n2min = a < b ? a : b, n2max = a > b ? a : b;
    bool ok = false;
    int bt = 0, bs = 0, ct = 0, cs = 0;
    if (n1max < n2min && cc == c1) {
      bt = b1; bs = b2; ct = c1; cs = c2; ok = true;
    }
    if (n2max < n1min && cc == c2) {
      bt = b2; bs = b1; ct = c2; cs = c1; ok = true;
    }
    if (!ok) return true;
    double nspt = k_max * P->del_t * (double)cn(bs, cs);
    double af = 1.0 / k_max;
    if (nspt < 1.0) return true;
    double min_tv = rad2vol(P->benv.frac, G->edges[bt - 1]);
    double max_sv = rad2vol(P->benv.frac, G->edges[bs]);
    double max_new = min_tv + max_sv * nspt;
    if (max_new / min_tv > 1.5) return true;
    for (int e = cn(bt, ct); e >= 1; e--) {
      int tp = ce(bt, ct, e);
      Tp target, src;
      load(tp, target);
      int ns, nc;
      if (!sample_source(bs, cs, target, nspt, af, &ns, &nc, src)) return false;
      if (nc > 0 && !target_with_source(bt, ct, e, src, cc)) return false;
      samp += ns;
      coag += nc;
    }
    *done = true;
    return true;
  }

  // mc_coag's bin-pair loop (coagulation.F90:72-94) with mc_coag_for_bin
  __device__ bool run() {
    if (R.rebuild && !sort_particles()) return false;
    for (int c1 = 1; c1 <= P->n_class; c1++)
      for (int c2 = 1; c2 <= c1; c2++)
        for (int b1 = 1; b1 <= nb; b1++) {
          if (cn(b1, c1) == 0) continue;
          int b2s = c1 == c2 ? b1 : 1;
          for (int b2 = b2s; b2 <= nb; b2++) {
            if (cn(b2, c2) == 0) continue;
            int cc = coag_dest_class(P->w, P->benv.frac, G->centers, b1 - 1, b2 - 1, c1 - 1, c2 - 1) + 1;
            double f_max =
                max_num_conc_factor(P->w, P->benv.frac, G->edges, b1 - 1, b2 - 1, c1 - 1, c2 - 1, cc - 1);
            double k_max = P->kmax_tab[(b1 - 1) + nb * (b2 - 1)] * f_max;
            bool done;
            if (!try_per_particle(k_max, b1, b2, c1, c2, cc, &done)) return false;
            if (done) continue;
            if (!per_set(k_max, b1, b2, c1, c2, cc)) return false;
          }
        }
    return true;
  }
};

__global__ void k_replay(const PopDev* pops, int pop, ReplayDev rd) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Seq s;
  s.P = &pops[pop];
  s.R = rd;
  s.g.u = rd.u;
  s.g.n = rd.n_u;
  s.g.pos = *rd.used;
  s.g.ok = true;
  s.n = *rd.n_part;
  s.status = 0;
  s.G = s.P->grid;
  s.nb = s.G->n_bin;
  s.samp = s.coag = 0;
  s.run();
  *rd.used = s.g.pos;
  *rd.n_part = s.n;
  *rd.status = s.status;
  rd.tot[0] = s.samp;
  rd.tot[1] = s.coag;
}

__global__ void k_replay_counts(RMapDev m, int* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m.n_r1 * m.n_r2) out[k] = m.inv_n[k];
}

}  // namespace

bool replay_reserve(ReplayBuffers& rb, int cap, int n_cells, int n_gc, int n_bin, int n_class,
                    int n_group) {
  size_t ints = 0;
  auto rm_ints = [&](int nc) { return (size_t)3 * cap + (size_t)nc + (size_t)nc * cap + 1; };
  ints = rm_ints(n_cells) + rm_ints(n_gc) + 8;
  size_t bytes = ints * sizeof(int) + 8 * sizeof(long long);
  if (rb.mem && rb.cap == cap && rb.n_cells == n_cells && rb.n_gc == n_gc) return true;
  replay_free(rb);
  if (cudaMalloc(&rb.mem, bytes) != cudaSuccess) {
    rb.mem = nullptr;
    return false;
  }
  cudaMemset(rb.mem, 0, bytes);
  rb.bytes = bytes;
  rb.cap = cap;
  rb.n_cells = n_cells;
  rb.n_gc = n_gc;
  rb.valid = false;
  long long* ll = (long long*)rb.mem;
  int* p = (int*)(ll + 8);
  auto carve = [&](RMapDev& m, int n1, int n2) {
    m.n_r1 = n1;
    m.n_r2 = n2;
    m.cap = cap;
    m.fwd1 = p; p += cap;
    m.fwd2 = p; p += cap;
    m.index = p; p += cap;
    m.inv_n = p; p += (size_t)n1 * n2;
    m.inv = p; p += (size_t)n1 * n2 * cap;
    m.n = p; p += 1;
  };
  carve(rb.dev.size_class, n_bin, n_class);
  carve(rb.dev.group_class, n_group, n_class);
  rb.dev.used = ll + 0;
  rb.dev.tot = ll + 1;  // [2]
  rb.dev.next_id = ll + 3;
  rb.dev.status = p;
  rb.dev.n_part = p + 1;
  return true;
}

void replay_free(ReplayBuffers& rb) {
  if (rb.mem) cudaFree(rb.mem);
  rb.mem = nullptr;
  rb.bytes = 0;
  rb.cap = rb.n_cells = rb.n_gc = 0;
  rb.valid = false;
}

void replay_launch(const PopDev* d_pops, int pop, const ReplayDev& rd, cudaStream_t stream) {
  k_replay<<<1, 32, 0, stream>>>(d_pops, pop, rd);
}

void replay_cell_counts(const ReplayDev& rd, int* d_counts, cudaStream_t stream) {
  int n = rd.size_class.n_r1 * rd.size_class.n_r2;
  if (n > 0) k_replay_counts<<<(n + 255) / 256, 256, 0, stream>>>(rd.size_class, d_counts);
}

}  // namespace pmc
