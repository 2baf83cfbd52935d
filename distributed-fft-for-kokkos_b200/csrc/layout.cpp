#include "layout.hpp"

namespace dfft {

std::vector<RankBlock> layout_blocks(const Layout& L) {
  const std::size_t P = L.nprocs(), D = L.gext.size();
  std::vector<RankBlock> blocks(P);
  std::size_t base = 0;
  for (std::size_t r = 0; r < P; ++r) {
    RankBlock& b = blocks[r];
    b.coords = rank_to_coord(L.topo, r, L.rank_right);
    b.starts = compute_local_starts(L.gext, L.topo, r, L.rank_right);
    b.local = compute_local_extents(L.gext, L.topo, identity_map(D), r, L.rank_right);
    b.mapped = compute_mapped_extents(L.pad.empty() ? b.local : L.pad, L.map);
    b.stride.assign(D, 0);
    std::size_t s = 1;
    if (L.view_right) {
      for (long i = static_cast<long>(D) - 1; i >= 0; --i) {
        b.stride[L.map[i]] = s;
        s *= b.mapped[i];
      }
    } else {
      for (std::size_t i = 0; i < D; ++i) {
        b.stride[L.map[i]] = s;
        s *= b.mapped[i];
      }
    }
    b.size = total_size(L.pad.empty() ? b.local : L.pad);
    b.base = base;
    base += b.size;
  }
  return blocks;
}

std::size_t layout_elements(const Layout& L) {
  return L.pad.empty() ? total_size(L.gext) : L.nprocs() * total_size(L.pad);
}

bool layout_even(const Layout& L) {
  for (std::size_t k = 0; k < L.gext.size(); ++k)
    if (L.topo[k] > 1 && L.gext[k] % L.topo[k] != 0) return false;
  return true;
}

// Padded blocks share one set of strides and one block size, so the offset
// splits into per-axis terms even when the bins are ragged.
bool layout_separable(const Layout& L) { return !L.pad.empty() || layout_even(L); }

std::size_t layout_fast_axis(const Layout& L) { return L.view_right ? L.map.back() : L.map.front(); }

LayoutTables build_layout_tables(const Layout& L) {
  LayoutTables T;
  const std::size_t D = L.gext.size(), P = L.nprocs();
  T.nd = static_cast<int>(D);
  auto blocks = layout_blocks(L);
  // stride of each axis in the rank numbering
  Ext rs(D, 1);
  std::size_t s = 1;
  if (L.rank_right) {
    for (long k = static_cast<long>(D) - 1; k >= 0; --k) {
      rs[k] = s;
      s *= L.topo[k];
    }
  } else {
    for (std::size_t k = 0; k < D; ++k) {
      rs[k] = s;
      s *= L.topo[k];
    }
  }
  // bin index and local index of every coordinate along an axis
  auto bins_of_axis = [&](std::size_t k, std::vector<std::int64_t>& bin, std::vector<std::int64_t>& local) {
    const std::int64_t n = static_cast<std::int64_t>(L.gext[k]), t = static_cast<std::int64_t>(L.topo[k]);
    bin.assign(n, 0);
    local.assign(n, 0);
    for (std::int64_t b = 0; b < t; ++b) {
      std::int64_t st, len;
      bin_mapping(n, t, b, st, len);
      for (std::int64_t c = st; c < st + len; ++c) {
        bin[c] = b;
        local[c] = c - st;
      }
    }
  };
  std::vector<std::int64_t> bin, local;
  if (layout_separable(L)) {
    T.mode = 0;
    const RankBlock& b0 = blocks[0];
    for (std::size_t k = 0; k < D; ++k) {
      bins_of_axis(k, bin, local);
      T.off[k] = static_cast<std::int64_t>(T.data.size());
      for (std::size_t c = 0; c < L.gext[k]; ++c)
        T.data.push_back(bin[c] * static_cast<std::int64_t>(rs[k] * b0.size) +
                         local[c] * static_cast<std::int64_t>(b0.stride[k]));
    }
  } else {
    T.mode = 1;
    for (std::size_t k = 0; k < D; ++k) {
      bins_of_axis(k, bin, local);
      T.rk[k] = static_cast<std::int64_t>(T.data.size());
      for (std::size_t c = 0; c < L.gext[k]; ++c) T.data.push_back(bin[c] * static_cast<std::int64_t>(rs[k]));
      T.loc[k] = static_cast<std::int64_t>(T.data.size());
      T.data.insert(T.data.end(), local.begin(), local.end());
    }
    T.rbase = static_cast<std::int64_t>(T.data.size());
    for (std::size_t r = 0; r < P; ++r) T.data.push_back(static_cast<std::int64_t>(blocks[r].base));
    T.rstride = static_cast<std::int64_t>(T.data.size());
    for (std::size_t r = 0; r < P; ++r)
      for (int k = 0; k < kMaxRank; ++k)
        T.data.push_back(k < static_cast<int>(D) ? static_cast<std::int64_t>(blocks[r].stride[k]) : 0);
  }
  return T;
}

}  // namespace dfft
