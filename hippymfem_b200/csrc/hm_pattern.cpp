// Host sparsity-pattern build for general dof tables (any mesh, any dof numbering).
//
// Same arrays as the reference's patternbuild.build_tables
// (hippymfem/fem/patternbuild.py:209-253, passes in hippymfem/fem/_patternkernels.py):
// the entries of each row are gathered through the row's element runs, ordered by a
// packed (column code, arrival) key -- code 0 for the diagonal when the rows lead with
// it, column + 1 otherwise -- and one scan gives the row's distinct columns and each
// entry's position.  Rows are independent, so they are split over host threads.
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/hippymfem_b200.h"

namespace {

struct Grouped {
  std::vector<int64_t> rcount;       // runs before each row (nrow + 1)
  std::vector<int64_t> runs_of_row;  // run ids (e * ndt + a) grouped by row, ascending
};

int group_rows(const int64_t* tdofs, int64_t ne, int ndt, int64_t nrow, Grouped& g) {
  g.rcount.assign(nrow + 1, 0);
  const int64_t nrun = ne * ndt;
  for (int64_t t = 0; t < nrun; ++t) {
    const int64_t r = tdofs[t];
    if (r < 0 || r >= nrow) return HM_ERR_RANGE;
    g.rcount[r + 1] += 1;
  }
  for (int64_t r = 0; r < nrow; ++r) g.rcount[r + 1] += g.rcount[r];
  std::vector<int64_t> fill(g.rcount.begin(), g.rcount.end() - 1);
  g.runs_of_row.resize(nrun);
  for (int64_t t = 0; t < nrun; ++t) g.runs_of_row[fill[tdofs[t]]++] = t;
  return HM_OK;
}

// Order the rows [r0, r1): ucount[r] and, per entry, its position within its row.
void order_rows(const int64_t* cdofs, int ndt, int ndr, int64_t ncol, int diag_first,
                const Grouped& g, int64_t r0, int64_t r1, int64_t* ucount, int32_t* slot,
                int32_t* indices, const int32_t* indptr, int* bad) {
  std::vector<uint64_t> key;
  std::vector<int64_t> ent;
  for (int64_t r = r0; r < r1; ++r) {
    const int64_t m = (g.rcount[r + 1] - g.rcount[r]) * ndr;
    if (m == 0) { ucount[r] = 0; continue; }
    key.resize(m);
    ent.resize(m);
    int64_t q = 0;
    for (int64_t p = g.rcount[r]; p < g.rcount[r + 1]; ++p) {
      const int64_t t = g.runs_of_row[p];
      const int64_t e = t / ndt;
      const int64_t k0 = t * ndr;
      for (int b = 0; b < ndr; ++b) {
        const int64_t c = cdofs[e * ndr + b];
        if (c < 0 || c >= ncol) { *bad = 1; return; }
        const uint64_t code = (diag_first && c == r) ? 0 : (uint64_t)(c + 1);
        key[q] = (code << 20) | (uint64_t)q;  // q < 2^20 entries a row
        ent[q] = k0 + b;
        ++q;
      }
    }
    std::sort(key.begin(), key.end());
    int64_t pos = -1;
    uint64_t prev = ~0ull;
    const int64_t base = indptr ? indptr[r] : 0;
    for (int64_t s = 0; s < m; ++s) {
      const uint64_t code = key[s] >> 20;
      if (code != prev) {
        ++pos;
        prev = code;
        if (indices) indices[base + pos] = (int32_t)(code == 0 ? r : (int64_t)code - 1);
      }
      if (slot) slot[ent[key[s] & ((1u << 20) - 1)]] = (int32_t)(base + pos);
    }
    ucount[r] = pos + 1;
  }
}

template <typename F>
void parallel_rows(int64_t nrow, int nthreads, F&& f) {
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nrow < 4096) nt = 1;
  std::vector<std::thread> th;
  const int64_t chunk = (nrow + nt - 1) / nt;
  for (int i = 0; i < nt; ++i) {
    const int64_t a = i * chunk, b = std::min(nrow, a + chunk);
    if (a >= b) break;
    th.emplace_back([=, &f] { f(a, b); });
  }
  for (auto& t : th) t.join();
}

}  // namespace

extern "C" int hm_pattern_build(const int64_t* tdofs, const int64_t* cdofs, int64_t ne, int ndt,
                                int ndr, int64_t nrow, int64_t ncol, int diag_first, int nthreads,
                                int32_t* indptr, int32_t* indices, int64_t indices_capacity,
                                int32_t* slot, int64_t* nnz) {
  if (ne < 0 || ndt <= 0 || ndr <= 0 || nrow < 0 || ncol < 0 || !indptr || !nnz) return HM_ERR_ARG;
  if ((ne > 0 && (!tdofs || !cdofs)) || ((indices == nullptr) != (slot == nullptr))) return HM_ERR_ARG;
  if (ne * (int64_t)ndt * ndr > INT32_MAX) return HM_ERR_UNSUPPORTED;
  Grouped g;
  int rc = group_rows(tdofs, ne, ndt, nrow, g);
  if (rc) return rc;
  int64_t maxrun = 0;
  for (int64_t r = 0; r < nrow; ++r) maxrun = std::max(maxrun, g.rcount[r + 1] - g.rcount[r]);
  if (maxrun * ndr >= (1 << 20)) return HM_ERR_UNSUPPORTED;
  std::vector<int64_t> ucount(nrow, 0);
  int bad = 0;
  // pass 1: distinct columns per row -> indptr
  parallel_rows(nrow, nthreads, [&](int64_t a, int64_t b) {
    int lbad = 0;
    order_rows(cdofs, ndt, ndr, ncol, diag_first, g, a, b, ucount.data(), nullptr, nullptr, nullptr, &lbad);
    if (lbad) bad = 1;
  });
  if (bad) return HM_ERR_RANGE;
  int64_t acc = 0;
  indptr[0] = 0;
  for (int64_t r = 0; r < nrow; ++r) {
    acc += ucount[r];
    if (acc > INT32_MAX) return HM_ERR_UNSUPPORTED;
    indptr[r + 1] = (int32_t)acc;
  }
  *nnz = acc;
  if (!indices) return HM_OK;
  if (indices_capacity < acc) return HM_ERR_NOMEM;
  // pass 2: columns and slots at their final places
  parallel_rows(nrow, nthreads, [&](int64_t a, int64_t b) {
    int lbad = 0;
    order_rows(cdofs, ndt, ndr, ncol, diag_first, g, a, b, ucount.data(), slot, indices, indptr, &lbad);
    if (lbad) bad = 1;
  });
  return bad ? HM_ERR_RANGE : HM_OK;
}
