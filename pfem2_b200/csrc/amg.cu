// amg.cu -- host setup of the smoothed-aggregation multigrid hierarchy of
// the pressure systems (runs once per pfem2_setup; FP64 throughout).
//
// Per system: level 0 is the eliminated pressure matrix (Dirichlet and
// padding rows have no off-diagonal entries and stay out of every
// aggregate). Levels 1 and 2 aggregate the level below with the classic
// three-pass greedy rule (seed + all-free neighbourhood, attach leftovers to
// the best-connected neighbouring aggregate, group the rest), restricted to
// one solver tile so that restriction never leaves the block that owns the
// tile. Level 3 takes one aggregate per tile. P_l is the tentative
// (piecewise-constant) prolongator smoothed once by (I - w D^-1 A_l), the
// coarse operator is the Galerkin product P_l^T A_l P_l, and w = 4 / (3
// rho(D^-1 A_l)) with rho from 30 power iterations (x 1.05).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "amg.h"

namespace pfem2 {

namespace {

struct Csr {
  int n = 0, m = 0;
  std::vector<int> ptr{0}, col;
  std::vector<double> val;
};

Csr transpose(const Csr& A) {
  Csr T;
  T.n = A.m;
  T.m = A.n;
  T.ptr.assign(A.m + 1, 0);
  for (int c : A.col) T.ptr[c + 1]++;
  for (int i = 0; i < A.m; ++i) T.ptr[i + 1] += T.ptr[i];
  T.col.resize(A.col.size());
  T.val.resize(A.col.size());
  std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
  for (int i = 0; i < A.n; ++i)
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) {
      const int p = pos[A.col[e]]++;
      T.col[p] = i;
      T.val[p] = A.val[e];
    }
  return T;
}

// C = A B, rows with ascending columns, exact zeros dropped
Csr spgemm(const Csr& A, const Csr& B) {
  Csr C;
  C.n = A.n;
  C.m = B.m;
  C.ptr.assign(A.n + 1, 0);
  std::vector<int> mark(B.m, -1), list;
  std::vector<double> acc(B.m, 0.0);
  for (int i = 0; i < A.n; ++i) {
    list.clear();
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) {
      const int k = A.col[e];
      const double a = A.val[e];
      for (int f = B.ptr[k]; f < B.ptr[k + 1]; ++f) {
        const int j = B.col[f];
        if (mark[j] != i) {
          mark[j] = i;
          acc[j] = 0.0;
          list.push_back(j);
        }
        acc[j] += a * B.val[f];
      }
    }
    std::sort(list.begin(), list.end());
    for (int j : list)
      if (acc[j] != 0.0) {
        C.col.push_back(j);
        C.val.push_back(acc[j]);
      }
    C.ptr[i + 1] = (int)C.col.size();
  }
  return C;
}

// (I - w D^-1 A) P
Csr smooth(const Csr& A, const std::vector<double>& dinv, double w, const Csr& P) {
  const Csr AP = spgemm(A, P);
  Csr R;
  R.n = P.n;
  R.m = P.m;
  R.ptr.assign(P.n + 1, 0);
  for (int i = 0; i < P.n; ++i) {
    int a = P.ptr[i], b = AP.ptr[i];
    const int ae = P.ptr[i + 1], be = AP.ptr[i + 1];
    const double s = w * dinv[i];
    while (a < ae || b < be) {
      int j;
      double v;
      if (b >= be || (a < ae && P.col[a] < AP.col[b])) {
        j = P.col[a];
        v = P.val[a++];
      } else if (a >= ae || AP.col[b] < P.col[a]) {
        j = AP.col[b];
        v = -s * AP.val[b++];
      } else {
        j = P.col[a];
        v = P.val[a++] - s * AP.val[b++];
      }
      if (v != 0.0) {
        R.col.push_back(j);
        R.val.push_back(v);
      }
    }
    R.ptr[i + 1] = (int)R.col.size();
  }
  return R;
}

double rho_dinv_a(const Csr& A, const std::vector<double>& dinv) {
  const int n = A.n;
  std::vector<double> x(n), y(n);
  for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.5 * std::sin(0.7 * i + 0.3);
  double lam = 1.0;
  for (int it = 0; it < 30; ++it) {
    double nx = 0.0, ny = 0.0;
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) s += A.val[e] * x[A.col[e]];
      y[i] = dinv[i] * s;
      nx += x[i] * x[i];
      ny += y[i] * y[i];
    }
    if (!(ny > 0.0)) break;
    lam = std::sqrt(ny / nx);
    const double inv = 1.0 / std::sqrt(ny);
    for (int i = 0; i < n; ++i) x[i] = y[i] * inv;
  }
  return 1.05 * lam;
}

bool isolated(const Csr& A, int i) {
  for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e)
    if (A.col[e] != i && A.val[e] != 0.0) return false;
  return true;
}

// Three-pass greedy aggregation inside tiles; aggregates renumbered in tile
// order (stable). Rows without off-diagonal entries get -1.
int aggregate(const Csr& A, const std::vector<int>& tile, std::vector<int>& agg) {
  const int n = A.n;
  agg.assign(n, -1);
  auto strong = [&](int i, int e) {
    const int j = A.col[e];
    return j != i && A.val[e] != 0.0 && tile[j] == tile[i];
  };
  std::vector<int> seed_tile;
  int na = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool any = false, free = true;
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e)
      if (strong(i, e)) {
        any = true;
        if (agg[A.col[e]] >= 0) free = false;
      }
    if (!any || !free) continue;
    agg[i] = na;
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e)
      if (strong(i, e)) agg[A.col[e]] = na;
    seed_tile.push_back(tile[i]);
    ++na;
  }
  std::vector<int> join(n, -1);
  std::vector<std::pair<int, int>> cnt;
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    cnt.clear();
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) {
      if (!strong(i, e) || agg[A.col[e]] < 0) continue;
      const int a = agg[A.col[e]];
      bool found = false;
      for (auto& pc : cnt)
        if (pc.first == a) {
          pc.second++;
          found = true;
        }
      if (!found) cnt.push_back({a, 1});
    }
    int best = -1, bc = 0;
    for (auto& pc : cnt)
      if (pc.second > bc || (pc.second == bc && pc.first < best)) {
        best = pc.first;
        bc = pc.second;
      }
    join[i] = best;
  }
  for (int i = 0; i < n; ++i)
    if (join[i] >= 0) agg[i] = join[i];
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0 || isolated(A, i)) continue;
    agg[i] = na;
    for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e)
      if (strong(i, e) && agg[A.col[e]] < 0) agg[A.col[e]] = na;
    seed_tile.push_back(tile[i]);
    ++na;
  }
  std::vector<int> order(na), newid(na);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return seed_tile[a] < seed_tile[b]; });
  for (int k = 0; k < na; ++k) newid[order[k]] = k;
  for (int i = 0; i < n; ++i)
    if (agg[i] >= 0) agg[i] = newid[agg[i]];
  return na;
}

// one aggregate per group of `per` consecutive tiles, counted from tile t0
// (rows with off-diagonal entries only)
int tile_aggregate(const Csr& A, const std::vector<int>& tile, int t0, int per, std::vector<int>& agg) {
  agg.assign(A.n, -1);
  int na = 0, last = -1;
  for (int i = 0; i < A.n; ++i) {
    if (isolated(A, i)) continue;
    const int g = (tile[i] - t0) / per;
    if (g != last) {
      last = g;
      ++na;
    }
    agg[i] = na - 1;
  }
  return na;
}

struct Level {
  Csr A, J, P, Pt2;
  std::vector<double> dinv;
  std::vector<int> tile;
  double w = 0.0;
};

}  // namespace

bool spd_inverse(std::vector<double>& M, int n) {
  std::vector<double> L((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = M[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    L[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = M[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      L[(size_t)i * n + j] = s / d;
    }
  }
  std::vector<double> Li((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s -= L[(size_t)i * n + k] * Li[(size_t)k * n + j];
      Li[(size_t)i * n + j] = s / L[(size_t)i * n + i];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += Li[(size_t)k * n + i] * Li[(size_t)k * n + j];
      M[(size_t)i * n + j] = s;
      M[(size_t)j * n + i] = s;
    }
  return true;
}

pfem2_status mg_build(const Ctx& c, const std::vector<double>& A, const std::vector<int>& col,
                      const std::vector<int>& len, const std::vector<Tile>& tiles, const std::vector<int>& st0,
                      const std::vector<int>& bt0, bool split, int coarse_max, MgHost& H) {
  const int ni = (int)c.inst.size(), T = (int)tiles.size(), G = (int)bt0.size() - 1;
  H.split = split;
  const std::vector<int>& sp = c.h_sl_ptr;
  std::vector<std::vector<Level>> sysL(ni);
  std::vector<std::vector<double>> Einv(ni);
  std::vector<double> w0(ni);
  H.j0.assign(c.nell, 0.0);
  for (int s = 0; s < ni; ++s) {
    const int v0 = c.inst[s].v_off, n0 = c.inst[s].nv_pad;
    std::vector<Level>& L = sysL[s];
    L.resize(kMgLevels);
    // level 0 from the SELL layout
    Csr& A0 = L[0].A;
    A0.n = A0.m = n0;
    A0.ptr.assign(n0 + 1, 0);
    L[0].tile.assign(n0, -1);
    for (int t = st0[s]; t < st0[s + 1]; ++t)
      for (int sl = tiles[t].s0; sl < tiles[t].s1; ++sl)
        for (int l = 0; l < kSlice; ++l) L[0].tile[sl * kSlice + l - v0] = t;
    for (int i = 0; i < n0; ++i) {
      const int row = v0 + i, sl = row / kSlice, lane = row % kSlice;
      for (int j = 0; j < len[sl]; ++j) {
        const int e = sp[sl] + j * kSlice + lane;
        if ((j > 0 && col[e] == row) || A[e] == 0.0) continue;
        A0.col.push_back(col[e] - v0);
        A0.val.push_back(A[e]);
      }
      A0.ptr[i + 1] = (int)A0.col.size();
    }
    for (int l = 0; l < kMgLevels; ++l) {
      Level& V = L[l];
      const int n = V.A.n;
      if (n == 0) {
        set_error("amg: a pressure system has an empty coarse level");
        return PFEM2_MESH_ERROR;
      }
      V.dinv.assign(n, 0.0);
      for (int i = 0; i < n; ++i) {
        double d = 0.0;
        for (int e = V.A.ptr[i]; e < V.A.ptr[i + 1]; ++e)
          if (V.A.col[e] == i) d = V.A.val[e];
        if (!(d > 0.0)) {
          set_error("amg: a diagonal entry of the pressure matrix is not positive");
          return PFEM2_MESH_ERROR;
        }
        V.dinv[i] = 1.0 / d;
      }
      if (l == kMgLevels - 1) {
        std::vector<double> E((size_t)n * n, 0.0);
        for (int i = 0; i < n; ++i)
          for (int e = V.A.ptr[i]; e < V.A.ptr[i + 1]; ++e) E[(size_t)i * n + V.A.col[e]] = V.A.val[e];
        // symmetrise the Galerkin product's rounding
        for (int i = 0; i < n; ++i)
          for (int j = 0; j < i; ++j) {
            const double m = 0.5 * (E[(size_t)i * n + j] + E[(size_t)j * n + i]);
            E[(size_t)i * n + j] = E[(size_t)j * n + i] = m;
          }
        if (!spd_inverse(E, n)) {
          set_error("amg: the coarsest pressure operator is not SPD");
          return PFEM2_MESH_ERROR;
        }
        Einv[s] = std::move(E);
        break;
      }
      V.w = 4.0 / (3.0 * rho_dinv_a(V.A, V.dinv));
      H.w.push_back(V.w);
      // J = 2 w D^-1 - w^2 D^-1 A D^-1
      V.J = V.A;
      for (int i = 0; i < n; ++i)
        for (int e = V.J.ptr[i]; e < V.J.ptr[i + 1]; ++e) {
          const int j = V.J.col[e];
          V.J.val[e] = -V.w * V.w * V.dinv[i] * V.A.val[e] * V.dinv[j] + (i == j ? 2.0 * V.w * V.dinv[i] : 0.0);
        }
      std::vector<int> agg;
      // the coarsest level: groups of tiles, at most coarse_max unknowns per system
      const int ntl = st0[s + 1] - st0[s], per = (ntl + coarse_max - 1) / coarse_max;
      const int na = l < kMgLevels - 2 ? aggregate(V.A, V.tile, agg) : tile_aggregate(V.A, V.tile, st0[s], per, agg);
      if (na == 0) {
        set_error("amg: aggregation produced no coarse unknowns");
        return PFEM2_MESH_ERROR;
      }
      Csr Pt;
      Pt.n = n;
      Pt.m = na;
      Pt.ptr.assign(n + 1, 0);
      std::vector<int> ctile(na, -1);
      for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) {
          Pt.col.push_back(agg[i]);
          Pt.val.push_back(1.0);
          ctile[agg[i]] = V.tile[i];
        }
        Pt.ptr[i + 1] = (int)Pt.col.size();
      }
      V.P = smooth(V.A, V.dinv, V.w, Pt);
      V.Pt2 = smooth(V.A, V.dinv, V.w, V.P);
      L[l + 1].A = spgemm(transpose(V.P), spgemm(V.A, V.P));
      L[l + 1].tile = ctile;
    }
    w0[s] = L[0].w;
    // J_0 on the SELL pattern
    for (int i = 0; i < n0; ++i) {
      const int row = v0 + i, sl = row / kSlice, lane = row % kSlice;
      const double di = L[0].dinv[i], w = L[0].w;
      for (int j = 0; j < len[sl]; ++j) {
        const int e = sp[sl] + j * kSlice + lane;
        const int cc = col[e] - v0;
        double v = -w * w * di * A[e] * L[0].dinv[cc];
        if (j == 0) v += 2.0 * w * di;
        H.j0[e] = v;
      }
    }
  }
  // ---- global numbering: systems in order, dofs tile-ordered inside
  std::vector<std::vector<int>> goff(kMgLevels, std::vector<int>(ni + 1, 0));
  for (int l = 1; l < kMgLevels; ++l) {
    for (int s = 0; s < ni; ++s) goff[l][s + 1] = goff[l][s] + sysL[s][l].A.n;
    H.n[l] = goff[l][ni];
    H.toff[l].assign(T + 1, 0);
    H.lsys[l].resize(H.n[l]);
    for (int s = 0; s < ni; ++s) {
      const std::vector<int>& tl = sysL[s][l].tile;
      for (int a = 0; a < (int)tl.size(); ++a) {
        H.toff[l][tl[a] + 1]++;
        H.lsys[l][goff[l][s] + a] = s;
      }
    }
    for (int t = 0; t < T; ++t) H.toff[l][t + 1] += H.toff[l][t];
  }
  H.n[0] = c.nv;
  // ---- restrictions
  auto append_rows = [](const Csr& M, int coff, std::vector<int>& ptr, std::vector<int>& cl, std::vector<double>& vl) {
    if (ptr.empty()) ptr.push_back(0);
    for (int i = 0; i < M.n; ++i) {
      for (int e = M.ptr[i]; e < M.ptr[i + 1]; ++e) {
        cl.push_back(M.col[e] + coff);
        vl.push_back(M.val[e]);
      }
      ptr.push_back((int)cl.size());
    }
  };
  for (int s = 0; s < ni; ++s) {
    std::vector<Level>& L = sysL[s];
    append_rows(transpose(L[0].Pt2), c.inst[s].v_off, H.r01_ptr, H.r01_col, H.r01_val);
    if (split) {
      append_rows(transpose(L[1].Pt2), goff[1][s], H.q2_ptr, H.q2_col, H.q2_val);
    } else {
      const Csr P01 = spgemm(L[0].Pt2, L[1].Pt2);
      append_rows(transpose(P01), c.inst[s].v_off, H.r02_ptr, H.r02_col, H.r02_val);
    }
    H.sys_D3.push_back(L[3].A.n);
    H.sys_off3.push_back(goff[3][s]);
    H.sys_n2.push_back(L[2].A.n);
    H.sys_off2.push_back(goff[2][s]);
    H.dmax = std::max(H.dmax, L[3].A.n);
  }
  // the restriction not in use: empty rows
  if (split) H.r02_ptr.assign(H.n[2] + 1, 0);
  else H.q2_ptr.assign(H.n[2] + 1, 0);
  // ---- per-block lists
  std::vector<int> sys_of_tile(T);
  for (int s = 0; s < ni; ++s)
    for (int t = st0[s]; t < st0[s + 1]; ++t) sys_of_tile[t] = s;
  std::vector<int> loc1(H.n[1], -1), loc2(H.n[2], -1), loc3(H.n[3], -1);
  for (int l = 1; l <= 2; ++l) {
    H.blk_s[l].assign(1, 0);
    H.s_jptr[l].assign(1, 0);
    H.s_pptr[l].assign(1, 0);
  }
  H.blk_s3.assign(1, 0);
  H.blk_e.assign(1, 0);
  H.p0_ptr.assign(c.nslices + 1, 0);
  H.p0_len.assign(c.nslices, 0);
  std::vector<std::vector<int>> p0c(c.nslices);
  std::vector<std::vector<double>> p0v(c.nslices);
  for (int l = 1; l <= 2; ++l) H.lk[l].assign(H.n[l], 0);
  std::vector<std::vector<int>> g3_rows(H.n[3]);
  H.c3_blk.assign(1, 0);
  for (int b = 0; b < G; ++b) {
    const int t_lo = bt0[b], t_hi = bt0[b + 1];
    // systems of a block are consecutive; lists store the index among them
    const int sys_first = t_hi > t_lo ? sys_of_tile[t_lo] : 0;
    for (int l = 1; l <= 2; ++l)
      for (int g = H.toff[l][t_lo]; g < H.toff[l][t_hi]; ++g) H.lk[l][g] = H.lsys[l][g] - sys_first;
    if (t_hi > t_lo) {
      int n2 = 0;
      for (int s = sys_of_tile[t_lo]; s <= sys_of_tile[t_hi - 1]; ++s) n2 += sysL[s][2].A.n;
      H.b2max = std::max(H.b2max, n2);
    }
    // contributions of the own level-2 rows to b3 = Pt2^T b2: one row per
    // touched level-3 dof, columns = own level-2 rows (relative index)
    {
      const int o2lo = H.toff[2][t_lo], o2hi = H.toff[2][t_hi];
      std::vector<std::pair<int, std::pair<int, double>>> ent;  // (level-3 dof, (own row, value))
      for (int g = o2lo; g < o2hi; ++g) {
        const int s = H.lsys[2][g], a = g - goff[2][s];
        const Csr& P = sysL[s][2].Pt2;
        for (int e = P.ptr[a]; e < P.ptr[a + 1]; ++e) ent.push_back({goff[3][s] + P.col[e], {g - o2lo, P.val[e]}});
      }
      std::stable_sort(ent.begin(), ent.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      for (size_t k = 0; k < ent.size(); ++k) {
        if (k == 0 || ent[k].first != ent[k - 1].first) {
          const int d = ent[k].first;
          g3_rows[d].push_back((int)H.c3_lk.size());
          H.c3_lk.push_back(H.lsys[3][d] - sys_first);
          H.c3_ptr.push_back((int)H.c3_col.size());
        }
        H.c3_col.push_back(ent[k].second.first);
        H.c3_val.push_back(ent[k].second.second);
      }
      H.c3_blk.push_back((int)H.c3_lk.size());
    }
    // S1: own level-1 dofs, then the halo the level-0 prolongation reads
    std::vector<int> S1, S2, S3;
    for (int g = H.toff[1][t_lo]; g < H.toff[1][t_hi]; ++g) S1.push_back(g);
    std::vector<int> halo;
    for (int t = t_lo; t < t_hi; ++t) {
      const int s = sys_of_tile[t], v0 = c.inst[s].v_off;
      const Csr& P = sysL[s][0].Pt2;
      for (int row = tiles[t].s0 * kSlice; row < tiles[t].s1 * kSlice; ++row)
        for (int e = P.ptr[row - v0]; e < P.ptr[row - v0 + 1]; ++e) {
          const int g = goff[1][s] + P.col[e];
          if (g < H.toff[1][t_lo] || g >= H.toff[1][t_hi]) halo.push_back(g);
        }
    }
    std::sort(halo.begin(), halo.end());
    halo.erase(std::unique(halo.begin(), halo.end()), halo.end());
    S1.insert(S1.end(), halo.begin(), halo.end());
    for (int k = 0; k < (int)S1.size(); ++k) loc1[S1[k]] = k;
    for (int g : S1) {
      const int s = H.lsys[1][g];
      const Csr& P = sysL[s][1].Pt2;
      const int a = g - goff[1][s];
      for (int e = P.ptr[a]; e < P.ptr[a + 1]; ++e) S2.push_back(goff[2][s] + P.col[e]);
    }
    std::sort(S2.begin(), S2.end());
    S2.erase(std::unique(S2.begin(), S2.end()), S2.end());
    for (int k = 0; k < (int)S2.size(); ++k) loc2[S2[k]] = k;
    for (int g : S2) {
      const int s = H.lsys[2][g];
      const Csr& P = sysL[s][2].Pt2;
      const int a = g - goff[2][s];
      for (int e = P.ptr[a]; e < P.ptr[a + 1]; ++e) S3.push_back(goff[3][s] + P.col[e]);
    }
    std::sort(S3.begin(), S3.end());
    S3.erase(std::unique(S3.begin(), S3.end()), S3.end());
    for (int k = 0; k < (int)S3.size(); ++k) loc3[S3[k]] = k;
    // level-1 and level-2 entries: J rows (global columns), Pt rows (local columns)
    const std::vector<int>* Sl[3] = {nullptr, &S1, &S2};
    std::vector<int>* locn[3] = {nullptr, &loc2, &loc3};
    for (int l = 1; l <= 2; ++l) {
      for (int g : *Sl[l]) {
        const int s = H.lsys[l][g], a = g - goff[l][s];
        const Level& V = sysL[s][l];
        H.s_sys[l].push_back(s - sys_first);
        for (int e = V.J.ptr[a]; e < V.J.ptr[a + 1]; ++e) {
          // level 1: global ids into b1; level 2: the system's own index
          // into the block's shared copy of b2
          H.s_jcol[l].push_back((l == 1 ? goff[l][s] : 0) + V.J.col[e]);
          H.s_jval[l].push_back(V.J.val[e]);
        }
        H.s_jptr[l].push_back((int)H.s_jcol[l].size());
        for (int e = V.Pt2.ptr[a]; e < V.Pt2.ptr[a + 1]; ++e) {
          H.s_pcol[l].push_back((*locn[l])[goff[l + 1][s] + V.Pt2.col[e]]);
          H.s_pval[l].push_back(V.Pt2.val[e]);
        }
        H.s_pptr[l].push_back((int)H.s_pcol[l].size());
      }
      H.blk_s[l].push_back((int)H.s_sys[l].size());
    }
    H.s1max = std::max(H.s1max, (int)S1.size());
    H.s2max = std::max(H.s2max, (int)S2.size());
    H.s3max = std::max(H.s3max, (int)S3.size());
    // level-3 entries: the coarse-inverse rows of each system's entries,
    // stored transposed ([d][entry]) so that the entries read consecutive
    // shared-memory words
    int eb = 0;
    for (size_t a = 0; a < S3.size();) {
      const int s = H.lsys[3][S3[a]], D = H.sys_D3[s];
      size_t b = a;
      while (b < S3.size() && H.lsys[3][S3[b]] == s) ++b;
      const int n = (int)(b - a);
      for (size_t j = a; j < b; ++j) {
        H.s3_sys.push_back(s - sys_first);
        H.s3_eoff.push_back(eb + (int)(j - a));
        H.s3_estr.push_back(n);
      }
      for (int d = 0; d < D; ++d)
        for (size_t j = a; j < b; ++j) H.s3_E.push_back((float)Einv[s][(size_t)(S3[j] - goff[3][s]) * D + d]);
      eb += D * n;
      a = b;
    }
    H.blk_s3.push_back((int)H.s3_sys.size());
    H.blk_e.push_back((int)H.s3_E.size());
    H.emax = std::max(H.emax, eb);
    // level-0 prolongation rows of the block's slices
    for (int t = t_lo; t < t_hi; ++t) {
      const int s = sys_of_tile[t], v0 = c.inst[s].v_off;
      const Csr& P = sysL[s][0].Pt2;
      for (int sl = tiles[t].s0; sl < tiles[t].s1; ++sl) {
        int mx = 0;
        for (int l = 0; l < kSlice; ++l) {
          const int i = sl * kSlice + l - v0;
          mx = std::max(mx, P.ptr[i + 1] - P.ptr[i]);
        }
        H.p0_len[sl] = mx;
        p0c[sl].assign((size_t)mx * kSlice, 0);
        p0v[sl].assign((size_t)mx * kSlice, 0.0);
        for (int l = 0; l < kSlice; ++l) {
          const int i = sl * kSlice + l - v0;
          for (int e = P.ptr[i]; e < P.ptr[i + 1]; ++e) {
            const int j = e - P.ptr[i];
            p0c[sl][(size_t)j * kSlice + l] = loc1[goff[1][s] + P.col[e]];
            p0v[sl][(size_t)j * kSlice + l] = P.val[e];
          }
        }
      }
    }
    for (int g : S1) loc1[g] = -1;
    for (int g : S2) loc2[g] = -1;
    for (int g : S3) loc3[g] = -1;
  }
  H.c3_ptr.push_back((int)H.c3_col.size());
  H.g3_ptr.assign(1, 0);
  H.c3_pos.assign(H.c3_lk.size(), 0);
  for (int d = 0; d < H.n[3]; ++d) {
    int n = H.g3_ptr.back();
    for (int r : g3_rows[d]) H.c3_pos[r] = n++;
    H.g3_ptr.push_back(n);
  }
  for (int sl = 0; sl < c.nslices; ++sl) {
    H.p0_ptr[sl + 1] = H.p0_ptr[sl] + H.p0_len[sl] * kSlice;
    H.p0_col.insert(H.p0_col.end(), p0c[sl].begin(), p0c[sl].end());
    H.p0_val.insert(H.p0_val.end(), p0v[sl].begin(), p0v[sl].end());
  }
  return PFEM2_OK;
}

}  // namespace pfem2
