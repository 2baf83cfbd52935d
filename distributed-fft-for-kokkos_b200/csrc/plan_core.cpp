// Host-side planning: restatement of the reference's topology / extents /
// block-analysis logic with runtime ranks.  File references are relative to
// the reference's `distributed/src/`.
#include "plan_core.hpp"

#include <algorithm>
#include <set>
#include <sstream>

namespace dfft {

[[noreturn]] void fail(int code, const std::string& msg) { throw Error(code, msg); }

std::string ext_str(const Ext& e) {
  std::ostringstream os;
  os << "(";
  for (std::size_t i = 0; i < e.size(); ++i) os << (i ? "," : "") << e[i];
  os << ")";
  return os.str();
}

bool BlockInfo::operator==(const BlockInfo& o) const {
  return in_topology == o.in_topology && out_topology == o.out_topology && in_extents == o.in_extents &&
         out_extents == o.out_extents && buffer_extents == o.buffer_extents && in_map == o.in_map &&
         out_map == o.out_map && in_axis == o.in_axis && out_axis == o.out_axis && fft_dim == o.fft_dim &&
         comm_axis == o.comm_axis && block_type == o.block_type && block_idx == o.block_idx;
}

// ---------------------------------------------------------------------------
// Container helpers: KokkosFFT_Distributed_ContainerAnalyses.hpp
// ---------------------------------------------------------------------------
std::size_t total_size(const Ext& v) {
  std::size_t s = 1;
  for (auto x : v) s *= x;
  return s;
}

std::size_t count_non_ones(const Ext& v) {
  return static_cast<std::size_t>(std::count_if(v.begin(), v.end(), [](std::size_t x) { return x != 1; }));
}

std::vector<std::size_t> extract_different_indices(const Ext& a, const Ext& b) {
  if (a.size() != b.size()) fail(kErrInvalidTopology, "Containers must have the same size.");
  std::vector<std::size_t> d;
  for (std::size_t i = 0; i < a.size(); ++i)
    if (a[i] != b[i]) d.push_back(i);
  return d;
}

// ContainerAnalyses.hpp:64-81: the set of every value that appears in a or b.
std::vector<std::size_t> extract_different_value_set(const Ext& a, const Ext& b) {
  if (a.size() != b.size()) fail(kErrInvalidTopology, "Containers must have the same size.");
  std::set<std::size_t> s;
  for (std::size_t i = 0; i < a.size(); ++i) {
    s.insert(a[i]);
    s.insert(b[i]);
  }
  return std::vector<std::size_t>(s.begin(), s.end());
}

std::vector<std::size_t> extract_non_one_indices(const Ext& a, const Ext& b) {
  if (a.size() != b.size()) fail(kErrInvalidTopology, "Containers must have the same size.");
  std::vector<std::size_t> r;
  for (std::size_t i = 0; i < a.size(); ++i)
    if (a[i] != 1 || b[i] != 1) r.push_back(i);
  return r;
}

Ext extract_non_one_values(const Ext& a) {
  Ext r;
  for (auto x : a)
    if (x != 1) r.push_back(x);
  return r;
}

bool has_identical_non_ones(const Ext& non_ones) {
  if (count_non_ones(non_ones) < 2) return false;
  return non_ones.size() == 2 && std::set<std::size_t>(non_ones.begin(), non_ones.end()).size() == 1;
}

Ext swap_elements(const Ext& arr, std::size_t i, std::size_t j) {
  Ext r = arr;
  std::swap(r.at(i), r.at(j));
  return r;
}

// ContainerAnalyses.hpp:182-229
Ext merge_topology(const Ext& in, const Ext& out) {
  auto in_size = total_size(in), out_size = total_size(out);
  if (in_size != out_size) fail(kErrInvalidTopology, "Input and output topologies must have the same size.");
  if (in_size == 1) return in;
  auto diff = extract_different_indices(in, out);
  if (diff.size() != 2)
    fail(kErrInvalidTopology, "Input and output topologies must differ exactly two positions: in_topology " +
                                  ext_str(in) + ", out_topology " + ext_str(out));
  Ext merged = in;
  for (std::size_t i = 0; i < in.size(); ++i) merged[i] = std::max(in[i], out[i]);
  return merged;
}

// ContainerAnalyses.hpp:240-258
std::size_t diff_topology(const Ext& in, const Ext& out) {
  if (total_size(in) == 1 && total_size(out) == 1) return 1;
  auto diff = extract_different_indices(in, out);
  if (diff.size() != 1) fail(kErrInvalidTopology, "Input and output topologies must differ at exactly one position.");
  return std::max(in.at(diff[0]), out.at(diff[0]));
}

std::size_t get_index(const Ext& v, std::size_t value) {
  return static_cast<std::size_t>(std::find(v.begin(), v.end(), value) - v.begin());
}

static bool is_found(const Ext& v, std::size_t value) { return std::find(v.begin(), v.end(), value) != v.end(); }

static Ext reversed(const Ext& v) { return Ext(v.rbegin(), v.rend()); }

Ext identity_map(std::size_t rank) {
  Ext m(rank);
  for (std::size_t i = 0; i < rank; ++i) m[i] = i;
  return m;
}

Ext compute_mapped_extents(const Ext& extents, const Ext& map) {
  Ext r(extents.size());
  for (std::size_t i = 0; i < extents.size(); ++i) r[i] = extents.at(map.at(i));
  return r;
}

// ---------------------------------------------------------------------------
// Topologies: KokkosFFT_Distributed_Topologies.hpp
// ---------------------------------------------------------------------------
TopologyType to_topology_type(const Ext& topo) {
  if (total_size(topo) == 0) return TopologyType::Empty;
  switch (count_non_ones(topo)) {
    case 0: return TopologyType::Shared;
    case 1: return TopologyType::Slab;
    case 2: return TopologyType::Pencil;
    case 3: return TopologyType::Brick;
    default: return TopologyType::Invalid;
  }
}

TopologyType get_common_topology_type(const std::vector<Ext>& topos) {
  for (auto& t : topos)
    if (to_topology_type(t) == TopologyType::Empty) return TopologyType::Empty;
  for (auto t : {TopologyType::Shared, TopologyType::Slab, TopologyType::Pencil, TopologyType::Brick}) {
    bool all = true;
    for (auto& x : topos) all = all && (to_topology_type(x) == t);
    if (all) return t;
  }
  return TopologyType::Invalid;
}

void slab_in_out_axes(const Ext& in, const Ext& out, std::size_t& in_axis, std::size_t& out_axis) {
  if (total_size(in) != total_size(out))
    fail(kErrInvalidTopology, "Input and output topologies must have the same size.");
  if (!(to_topology_type(in) == TopologyType::Slab && to_topology_type(out) == TopologyType::Slab))
    fail(kErrInvalidTopology, "Input and output topologies must be slab topologies.");
  in_axis = 0;
  out_axis = 0;
  for (std::size_t i = 0; i < in.size(); ++i) {
    if (in[i] > 1 && out[i] == 1) out_axis = i;
    if (in[i] == 1 && out[i] > 1) in_axis = i;
  }
}

void pencil_in_out_axes(const Ext& in, const Ext& out, std::size_t& in_axis, std::size_t& out_axis) {
  auto in_size = total_size(in), out_size = total_size(out);
  if (in_size == 1 || out_size == 1)
    fail(kErrInvalidTopology, "Input and output topologies must have at least one non-trivial dimension.");
  if (in_size != out_size) fail(kErrInvalidTopology, "Input and output topologies must have the same size.");
  in_axis = 0;
  out_axis = 0;
  for (std::size_t i = 0; i < in.size(); ++i) {
    if (in[i] != out[i]) {
      if (in[i] == 1) in_axis = i;
      if (out[i] == 1) out_axis = i;
    }
  }
}

// Topologies.hpp:191-242
Ext propose_mid_array(const Ext& in, const Ext& out) {
  auto diff_indices = extract_different_indices(in, out);
  auto diff_value_set = extract_different_value_set(in, out);
  auto diff_non_one_indices = extract_non_one_indices(in, out);
  if (diff_non_one_indices.size() < 3)
    fail(kErrInvalidTopology,
         "The total number of non-one elements either in Input and output topologies must be three.");
  if (diff_indices.size() < 3 && diff_value_set.size() == 3)
    fail(kErrInvalidTopology, "Input and output topologies must differ exactly three positions.");
  Ext in_trimmed(in.size(), 0), out_trimmed(out.size(), 0);
  for (auto d : diff_indices) {
    in_trimmed.at(d) = in.at(d);
    out_trimmed.at(d) = out.at(d);
  }
  std::size_t idx_one_in = get_index(in_trimmed, 1);
  std::size_t idx_one_out = get_index(out_trimmed, 1);
  for (std::size_t i = 0; i < diff_non_one_indices.size(); ++i) {
    for (std::size_t j = i + 1; j < diff_non_one_indices.size(); ++j) {
      std::size_t idx_in = diff_non_one_indices.at(i), idx_out = diff_non_one_indices.at(j);
      Ext mid = swap_elements(in, idx_in, idx_out);
      std::size_t idx_one_mid = get_index(mid, 1);
      auto mid_in = extract_different_indices(mid, in);
      auto mid_out = extract_different_indices(mid, out);
      if (mid_in.size() == 2 && mid_out.size() == 2 && !(idx_one_mid == idx_one_in || idx_one_mid == idx_one_out)) {
        auto a0 = mid.at(mid_in.at(0)), a1 = mid.at(mid_in.at(1));
        auto b0 = mid.at(mid_out.at(0)), b1 = mid.at(mid_out.at(1));
        if ((a0 == 1 || a1 == 1) && (b0 == 1 || b1 == 1)) return mid;
      }
    }
  }
  return out;
}

// Topologies.hpp:259-331
std::vector<std::vector<std::size_t>> decompose_axes(const std::vector<Ext>& topos, const Ext& axes) {
  Ext axes_reversed = reversed(axes);
  std::vector<std::vector<std::size_t>> all_axes;
  for (auto& topo : topos) {
    Ext ready;
    for (auto axis : axes_reversed) {
      if (topo.at(axis) > 1) break;
      ready.push_back(axis);
    }
    all_axes.push_back(reversed(ready));
    for (auto axis : ready) {
      auto it = std::find(axes_reversed.begin(), axes_reversed.end(), axis);
      if (it != axes_reversed.end()) axes_reversed.erase(it);
    }
  }
  std::size_t total = 0;
  for (auto& a : all_axes) total += a.size();
  if (total != axes.size()) fail(kErrInvalidTopology, "Axes are not decomposed correctly");
  return all_axes;
}

// Topologies.hpp:352-399
std::size_t compute_trans_axis(const Ext& in, const Ext& out, std::size_t first_non_one) {
  auto in_non_ones = extract_non_one_values(in);
  auto out_non_ones = extract_non_one_values(out);
  std::string topo_msg = "in_topology " + ext_str(in) + ", out_topology " + ext_str(out);
  if (in_non_ones.size() != 2 || out_non_ones.size() != 2)
    fail(kErrInvalidTopology, "Input and output topologies must have exactly two non-one elements. " + topo_msg);
  if (has_identical_non_ones(in_non_ones) || has_identical_non_ones(out_non_ones))
    fail(kErrInvalidTopology, "Input and output topologies must not have identical non-one elements. " + topo_msg);
  auto diff = extract_different_indices(in, out);
  if (diff.size() != 2)
    fail(kErrInvalidTopology, "Input and output topologies must differ exactly two positions " + topo_msg);
  std::size_t exchange_non_one = 0;
  for (auto d : diff) {
    if (in.at(d) > 1) {
      exchange_non_one = in.at(d);
      break;
    }
  }
  return !(exchange_non_one == first_non_one) ? 1 : 0;
}

// Topologies.hpp:421-618
std::vector<Ext> get_all_slab_topologies(const Ext& in, const Ext& out, const Ext& axes) {
  const std::size_t DIM = in.size(), FFT_DIM = axes.size();
  if (!(FFT_DIM >= 1 && FFT_DIM <= 3)) fail(kErrInvalidArgument, "FFT_DIM must be in [1, 3]");
  if (!(DIM >= 2 && DIM >= FFT_DIM)) fail(kErrInvalidArgument, "DIM >= 2 and DIM >= FFT_DIM");
  if (!(to_topology_type(in) == TopologyType::Slab && to_topology_type(out) == TopologyType::Slab))
    fail(kErrInvalidTopology, "Input and output topologies must be slab topologies.");

  std::vector<Ext> topologies{in};
  const std::size_t p = total_size(in);
  auto add_topology_at = [&](std::size_t axis) {
    Ext t(DIM, 1);
    t.at(axis) = p;
    if (topologies.back() != t) topologies.push_back(t);
  };
  auto add_topology_at_first_one = [&](const Ext& topo) {
    for (std::size_t i = 0; i < DIM; ++i) {
      if (topo.at(i) == 1) {
        add_topology_at(i);
        break;
      }
    }
  };
  auto finalize = [&]() {
    if (topologies.back() != out) topologies.push_back(out);
    return topologies;
  };

  if (DIM == 2 && FFT_DIM == 2) {
    if (in == out) {
      add_topology_at_first_one(in);
    } else {
      auto last_axis = axes.back();
      if (in.at(last_axis) != 1) {
        add_topology_at_first_one(in);
        if (topologies.back() != in) topologies.push_back(in);
      }
    }
    return finalize();
  }

  if (DIM == 3 && FFT_DIM == 3) {
    auto last_axis = axes.back();
    auto first_dim = in.at(last_axis);
    if (in == out) {
      if (first_dim != 1) add_topology_at(axes.at(0));
      else add_topology_at(axes.back());
    } else {
      if (first_dim != 1) {
        add_topology_at(axes.at(0));
        if (out.at(axes.front()) != 1) add_topology_at_first_one(topologies.back());
      } else {
        if (in.at(axes.at(1)) != 1) {
          add_topology_at(axes.back());
        } else {
          if (out.at(axes.front()) != 1) add_topology_at_first_one(topologies.back());
        }
      }
    }
    return finalize();
  }

  // Batched case
  Ext axes_reversed = axes;
  auto is_topology_ready = [&](const Ext& topo) {
    bool ready = true;
    for (auto axis : axes_reversed)
      if (topo.at(axis) > 1) ready = false;
    return ready;
  };
  if (is_topology_ready(in) || is_topology_ready(out)) return finalize();

  if (FFT_DIM == 1) {
    for (std::size_t i = 0; i < DIM; ++i) {
      if (!is_found(axes_reversed, i)) {
        add_topology_at(i);
        break;
      }
    }
    return finalize();
  } else if (DIM > 3 && FFT_DIM == 3) {
    Ext sorted_axes = axes;
    std::sort(sorted_axes.begin(), sorted_axes.end());
    std::reverse(axes_reversed.begin(), axes_reversed.end());
    Ext ready;
    for (auto axis : axes_reversed) {
      if (in.at(axis) > 1) break;
      ready.push_back(axis);
    }
    if (ready.empty()) {
      add_topology_at(axes_reversed.back());
      for (auto axis : axes_reversed) {
        if (topologies.back().at(axis) > 1) break;
        ready.push_back(axis);
      }
    }
    for (auto axis : ready) {
      auto it = std::find(axes_reversed.begin(), axes_reversed.end(), axis);
      if (it != axes_reversed.end()) axes_reversed.erase(it);
    }
    if (!is_topology_ready(out)) {
      for (auto axis : sorted_axes) {
        if (!is_found(axes_reversed, axis)) {
          add_topology_at(axis);
          break;
        }
      }
    }
    return finalize();
  } else {
    std::reverse(axes_reversed.begin(), axes_reversed.end());
    Ext ready;
    for (auto axis : axes_reversed) {
      if (in.at(axis) > 1) break;
      ready.push_back(axis);
    }
    for (auto axis : ready) {
      auto it = std::find(axes_reversed.begin(), axes_reversed.end(), axis);
      if (it != axes_reversed.end()) axes_reversed.erase(it);
    }
    if (!is_topology_ready(out)) {
      for (std::size_t i = 0; i < DIM; ++i) {
        if (!is_found(axes_reversed, i)) {
          add_topology_at(i);
          break;
        }
      }
    }
    return finalize();
  }
}

// Topologies.hpp:645-811
PencilChain get_all_pencil_topologies(const Ext& in_topology, bool in_right, const Ext& out_topology, bool out_right,
                                      const Ext& axes) {
  const std::size_t DIM = in_topology.size(), FFT_DIM = axes.size();
  if (!(FFT_DIM >= 1 && FFT_DIM <= 3)) fail(kErrInvalidArgument, "FFT_DIM must be in [1, 3]");
  if (!(DIM >= 3 && DIM >= FFT_DIM)) fail(kErrInvalidArgument, "DIM >= 3 and DIM >= FFT_DIM");
  if (!(to_topology_type(in_topology) == TopologyType::Pencil &&
        to_topology_type(out_topology) == TopologyType::Pencil))
    fail(kErrInvalidTopology, "Input and output topologies must be pencil topologies.");

  Ext axes_reversed = axes;
  Ext non_ones = extract_non_one_values(in_topology);
  bool has_same_non_one_elements = has_identical_non_ones(non_ones);
  Ext in_tmp = in_topology, out_tmp = out_topology;

  if (has_same_non_one_elements) {
    // Equal px == py: relabel the two non-one entries by dummies 2, 3 so that
    // the exchanges can be told apart (Topologies.hpp:671-692).
    Ext dummies{2, 3};
    std::size_t count = 0;
    for (std::size_t i = 0; i < DIM; ++i)
      if (in_tmp[i] > 1) in_tmp[i] = dummies.at(count++);
    count = 0;
    if (in_right != out_right) std::reverse(dummies.begin(), dummies.end());
    for (std::size_t i = 0; i < DIM; ++i)
      if (out_tmp[i] > 1) out_tmp[i] = dummies.at(count++);
  }

  const std::size_t first_non_one =
      in_right ? extract_non_one_values(in_tmp).at(0) : extract_non_one_values(in_tmp).at(1);

  PencilChain ch;
  auto get_layout = [&](const Ext& t) -> std::size_t {
    return extract_non_one_values(t).at(0) == first_non_one ? 1 : 0;
  };
  auto to_original = [&]() {
    if (has_same_non_one_elements) {
      auto v = non_ones.at(0);
      for (auto& t : ch.topologies)
        for (auto& x : t)
          if (x > 1) x = v;
    }
    return ch;
  };

  ch.topologies.push_back(in_tmp);
  ch.layouts.push_back(get_layout(in_tmp));

  auto add_topology = [&](const Ext& topo) {
    if (ch.topologies.back() != topo) {
      ch.trans_axes.push_back(compute_trans_axis(ch.topologies.back(), topo, first_non_one));
      ch.topologies.push_back(topo);
      ch.layouts.push_back(get_layout(topo));
    }
  };
  auto try_add_mid_topology = [&]() {
    try {
      auto mid = propose_mid_array(ch.topologies.back(), out_tmp);
      add_topology(mid);
    } catch (std::runtime_error&) {
    }
  };
  auto finalize = [&]() {
    add_topology(out_tmp);
    return to_original();
  };
  auto is_topology_ready = [&](const Ext& topo, const Ext& cur_axes) {
    for (auto axis : cur_axes)
      if (topo.at(axis) != 1) return false;
    return true;
  };

  if (is_topology_ready(in_tmp, axes_reversed) || is_topology_ready(out_tmp, axes_reversed)) {
    try_add_mid_topology();
    return finalize();
  }

  std::reverse(axes_reversed.begin(), axes_reversed.end());
  Ext shuffled = in_tmp;
  auto last_axis = axes_reversed.front();
  auto first_axis = axes_reversed.back();
  auto first_dim = in_tmp.at(last_axis);
  auto last_dim = out_tmp.at(first_axis);
  if (first_dim == 1) axes_reversed.erase(axes_reversed.begin());
  if (last_dim == 1 && !axes_reversed.empty()) axes_reversed.pop_back();

  for (auto axis : axes_reversed) {
    std::size_t swap_idx = 0;
    if (in_tmp == out_tmp) {
      for (std::size_t idx = 0; idx < DIM; ++idx) {
        if (shuffled.at(idx) == 1 && idx != axis) {
          swap_idx = idx;
          break;
        }
      }
    } else {
      auto diff_non_one = extract_non_one_indices(in_tmp, out_tmp);
      for (auto d : diff_non_one) {
        if (shuffled.at(d) == 1 && d != axis) {
          swap_idx = d;
          break;
        }
      }
    }
    shuffled = swap_elements(shuffled, axis, swap_idx);
    add_topology(shuffled);
  }

  if (ch.topologies.back() == out_tmp) return to_original();
  try_add_mid_topology();
  return finalize();
}

// ---------------------------------------------------------------------------
// Layout math
// ---------------------------------------------------------------------------
void bin_mapping(std::int64_t n, std::int64_t nbins, std::int64_t ibin, std::int64_t& start, std::int64_t& length) {
  std::int64_t base = n / nbins, rem = n % nbins;
  length = base + (ibin < rem ? 1 : 0);
  start = ibin * base + std::min(ibin, rem);
}

Ext rank_to_coord(const Ext& topology, std::size_t rank, bool layout_right) {
  Ext coord(topology.size(), 0);
  if (rank >= total_size(topology)) fail(kErrInvalidArgument, "rank must be less than topology size.");
  std::size_t r = rank;
  const long nd = static_cast<long>(topology.size());
  if (layout_right) {
    for (long i = nd - 1; i >= 0; --i) {
      coord[i] = r % topology[i];
      r /= topology[i];
    }
  } else {
    for (long i = 0; i < nd; ++i) {
      coord[i] = r % topology[i];
      r /= topology[i];
    }
  }
  return coord;
}

Ext compute_local_extents(const Ext& extents, const Ext& topology, const Ext& map, std::size_t rank,
                          bool layout_right) {
  Ext local = extents;
  auto coords = rank_to_coord(topology, rank, layout_right);
  for (std::size_t i = 0; i < extents.size(); ++i) {
    if (topology.at(i) > 1) {
      std::size_t n = extents[i], t = topology[i];
      local[i] = (coords[i] < n % t) ? n / t + 1 : n / t;
    }
  }
  return compute_mapped_extents(local, map);
}

Ext compute_local_starts(const Ext& extents, const Ext& topology, std::size_t rank, bool layout_right) {
  Ext starts(extents.size(), 0);
  auto coords = rank_to_coord(topology, rank, layout_right);
  for (std::size_t i = 0; i < extents.size(); ++i) {
    if (topology[i] > 1) {
      std::int64_t s, l;
      bin_mapping(static_cast<std::int64_t>(extents[i]), static_cast<std::int64_t>(topology[i]),
                  static_cast<std::int64_t>(coords[i]), s, l);
      starts[i] = static_cast<std::size_t>(s);
    }
  }
  return starts;
}

Ext compute_buffer_extents(const Ext& extents, const Ext& in_topo, const Ext& out_topo, bool view_layout_right) {
  Ext merged = merge_topology(in_topo, out_topo);
  std::size_t p0 = diff_topology(merged, in_topo);
  Ext buf(extents.size() + 1);
  if (view_layout_right) {
    buf[0] = p0;
    for (std::size_t i = 0; i < extents.size(); ++i) buf[i + 1] = (extents[i] - 1) / merged[i] + 1;
  } else {
    for (std::size_t i = 0; i < extents.size(); ++i) buf[i] = (extents[i] - 1) / merged[i] + 1;
    buf.back() = p0;
  }
  return buf;
}

Ext compute_fft_extents(const Ext& in_extents, const Ext& out_extents, const Ext& axes) {
  Ext r;
  for (auto a : axes) r.push_back(std::max(in_extents.at(a), out_extents.at(a)));
  return r;
}

Ext permute_map_by_axes(const Ext& src_map, const Ext& axes, bool view_layout_right) {
  Ext map;
  if (view_layout_right) {
    for (auto s : src_map)
      if (!is_found(axes, s)) map.push_back(s);
    for (auto a : axes) map.push_back(a);
  } else {
    Ext ar = reversed(axes);
    for (auto a : ar) map.push_back(a);
    for (auto s : src_map)
      if (!is_found(ar, s)) map.push_back(s);
  }
  map.resize(src_map.size());
  return map;
}

Ext get_map_axes(std::size_t rank, const Ext& axes, bool view_layout_right) {
  return permute_map_by_axes(identity_map(rank), axes, view_layout_right);
}

// ---------------------------------------------------------------------------
// Block analyses: KokkosFFT_Distributed_BlockAnalyses.hpp
// ---------------------------------------------------------------------------
namespace {

std::size_t count_blocks(const std::vector<BlockInfo>& b, BlockType t) {
  return static_cast<std::size_t>(
      std::count_if(b.begin(), b.end(), [t](const BlockInfo& x) { return x.block_type == t; }));
}

std::size_t count_fft_dims(const std::vector<BlockInfo>& b) {
  std::size_t s = 0;
  for (auto& x : b)
    if (x.block_type == BlockType::FFT) s += x.fft_dim;
  return s;
}

struct Proposal {
  BlockInfo block;
  std::size_t max_buffer_size;
};

// BlockAnalyses.hpp:55-72
Proposal propose_fft_block(const Ext& map, const Ext& in_extents, const Ext& out_extents, std::size_t fft_dim,
                           std::size_t block_idx) {
  BlockInfo b;
  b.block_type = BlockType::FFT;
  b.fft_dim = fft_dim;
  b.in_extents = in_extents;
  b.out_extents = out_extents;
  b.in_map = map;
  b.out_map = map;
  b.block_idx = block_idx;
  const std::size_t rank = map.size();
  b.in_topology.assign(rank, 0);
  b.out_topology.assign(rank, 0);
  b.buffer_extents.assign(rank + 1, 0);
  return {b, total_size(out_extents) * 2};
}

// BlockAnalyses.hpp:93-136
Proposal propose_transpose_block(const Ext& map, const Ext& in_topo, const Ext& out_topo, const Ext& in_extents,
                                 const Ext& global_extents, const Ext& axes, std::size_t rank, bool is_layout_right,
                                 bool is_last, std::size_t in_axis, std::size_t out_axis, std::size_t comm_axis,
                                 std::size_t block_idx, std::size_t size_factor, bool view_layout_right) {
  BlockInfo b;
  b.block_type = BlockType::Transpose;
  b.in_map = map;
  b.in_axis = in_axis;
  b.out_axis = out_axis;
  b.comm_axis = comm_axis;
  b.in_topology = in_topo;
  b.out_topology = out_topo;
  b.in_extents = in_extents;
  b.block_idx = block_idx;
  if (is_last) {
    b.out_map = identity_map(map.size());
  } else {
    b.out_map = axes.empty() ? permute_map_by_axes(b.in_map, Ext{out_axis}, view_layout_right)
                             : permute_map_by_axes(b.in_map, axes, view_layout_right);
  }
  b.out_extents = compute_local_extents(global_extents, out_topo, b.out_map, rank, is_layout_right);
  b.buffer_extents = compute_buffer_extents(global_extents, in_topo, out_topo, view_layout_right);
  std::size_t mx = std::max({total_size(b.in_extents), total_size(b.buffer_extents), total_size(b.out_extents)});
  return {b, mx * size_factor};
}

struct ProposeContext {
  bool pencil;
  bool view_layout_right;
  bool real_input;
  std::size_t fft_rank;  // FFT_DIM
  const Ext* in_extents;
  const Ext* gin;
  const Ext* gout;
  const std::vector<Ext>* topologies;
  const std::vector<std::size_t>* trans_axes;  // pencil only
  const std::vector<std::size_t>* layouts;     // pencil only
  const std::vector<std::vector<std::size_t>>* all_axes;
  const Ext* map;
  std::size_t rank;
};

// BlockAnalyses.hpp:157-258 (slab) and :281-388 (pencil); the two differ only
// in the in/out-axis helper, the comm axis and the rank-order flags.
std::vector<Proposal> propose_block(const ProposeContext& c, const std::vector<BlockInfo>& infos,
                                    std::size_t block_idx) {
  const auto& topos = *c.topologies;
  auto compute_transpose_block = [&](const std::vector<BlockInfo>& bi, std::size_t size_factor) {
    bool is_last = block_idx == (topos.size() - 1);
    std::size_t nb_trans = count_blocks(bi, BlockType::Transpose);
    const Ext& cur = topos.at(nb_trans);
    const Ext& next = topos.at(nb_trans + 1);
    std::size_t in_axis, out_axis;
    if (c.pencil) pencil_in_out_axes(cur, next, in_axis, out_axis);
    else slab_in_out_axes(cur, next, in_axis, out_axis);
    Ext next_axes;
    if (!is_last) next_axes.assign(c.all_axes->at(block_idx + 1).begin(), c.all_axes->at(block_idx + 1).end());
    std::size_t comm_axis = c.pencil ? c.trans_axes->at(nb_trans) : 0;
    bool is_layout_right = c.pencil ? (c.layouts->at(nb_trans + 1) != 0) : true;
    if (bi.empty()) {
      return propose_transpose_block(identity_map(c.map->size()), cur, next, *c.in_extents, *c.gin, next_axes,
                                     c.rank, is_layout_right, false, in_axis, out_axis, comm_axis, 0, size_factor,
                                     c.view_layout_right);
    }
    return propose_transpose_block(bi.back().out_map, cur, next, bi.back().out_extents, *c.gout, next_axes, c.rank,
                                   is_layout_right, is_last, in_axis, out_axis, comm_axis, nb_trans, 2,
                                   c.view_layout_right);
  };

  std::vector<Proposal> out;
  const auto& axes = c.all_axes->at(block_idx);
  const std::size_t fft_dim = axes.size();
  if (fft_dim == 0) {
    out.push_back(compute_transpose_block(infos, c.real_input ? 1 : 2));
    return out;
  }
  bool is_layout_right = c.pencil ? (c.layouts->at(block_idx) != 0) : true;
  bool is_last_fft_block = (count_fft_dims(infos) + fft_dim) == c.fft_rank;
  if (infos.empty()) {
    const Ext& topology = topos.at(block_idx);
    Ext fin = compute_mapped_extents(*c.in_extents, *c.map);
    Ext fout = compute_local_extents(*c.gout, topology, *c.map, c.rank, is_layout_right);
    out.push_back(propose_fft_block(*c.map, fin, fout, fft_dim, 0));
    if (!is_last_fft_block) {
      auto nb = infos;
      nb.push_back(out.back().block);
      out.push_back(compute_transpose_block(nb, 2));
    }
    return out;
  }
  std::size_t nb_fft = count_blocks(infos, BlockType::FFT);
  const Ext in_map = infos.back().out_map;
  const Ext fin = infos.back().out_extents;
  if (nb_fft == 0) {
    const Ext topology = infos.back().out_topology;
    Ext fout = compute_local_extents(*c.gout, topology, in_map, c.rank, is_layout_right);
    out.push_back(propose_fft_block(in_map, fin, fout, fft_dim, 0));
  } else {
    out.push_back(propose_fft_block(in_map, fin, fin, fft_dim, nb_fft));
  }
  if (!is_last_fft_block) {
    auto nb = infos;
    nb.push_back(out.back().block);
    out.push_back(compute_transpose_block(nb, 2));
  }
  return out;
}

}  // namespace

BlockInfo propose_transpose(const Ext& map, const Ext& in_topo, const Ext& out_topo, const Ext& in_extents,
                            const Ext& global_extents, const Ext& axes, std::size_t rank, bool is_layout_right,
                            bool is_last, std::size_t in_axis, std::size_t out_axis, std::size_t comm_axis,
                            std::size_t block_idx, std::size_t size_factor, bool view_layout_right,
                            std::size_t* max_buffer_size) {
  const Proposal p = propose_transpose_block(map, in_topo, out_topo, in_extents, global_extents, axes, rank,
                                             is_layout_right, is_last, in_axis, out_axis, comm_axis, block_idx,
                                             size_factor, view_layout_right);
  if (max_buffer_size) *max_buffer_size = p.max_buffer_size;
  return p.block;
}

BlockAnalyses slab_block_analyses(const Ext& in_extents, const Ext& gin, const Ext& gout, const Ext& in_topo,
                                  const Ext& out_topo, const Ext& axes, bool real_input, bool view_layout_right,
                                  std::size_t rank) {
  Ext map = get_map_axes(in_topo.size(), axes, view_layout_right);
  auto topologies = get_all_slab_topologies(in_topo, out_topo, axes);
  auto all_axes = decompose_axes(topologies, axes);
  ProposeContext c{false, view_layout_right, real_input, axes.size(), &in_extents, &gin, &gout,
                   &topologies, nullptr, nullptr, &all_axes, &map, rank};
  BlockAnalyses r;
  for (std::size_t it = 0; it < topologies.size(); ++it) {
    for (auto& p : propose_block(c, r.blocks, it)) {
      r.blocks.push_back(p.block);
      r.max_buffer_size = std::max(r.max_buffer_size, p.max_buffer_size);
    }
  }
  return r;
}

BlockAnalyses pencil_block_analyses(const Ext& in_extents, const Ext& gin, const Ext& gout, const Ext& in_topo,
                                    bool in_right, const Ext& out_topo, bool out_right, const Ext& axes,
                                    bool real_input, bool view_layout_right, std::size_t rank) {
  Ext map = get_map_axes(in_topo.size(), axes, view_layout_right);
  auto ch = get_all_pencil_topologies(in_topo, in_right, out_topo, out_right, axes);
  auto all_axes = decompose_axes(ch.topologies, axes);
  ProposeContext c{true, view_layout_right, real_input, axes.size(), &in_extents, &gin, &gout,
                   &ch.topologies, &ch.trans_axes, &ch.layouts, &all_axes, &map, rank};
  BlockAnalyses r;
  for (std::size_t it = 0; it < ch.topologies.size(); ++it) {
    for (auto& p : propose_block(c, r.blocks, it)) {
      r.blocks.push_back(p.block);
      r.max_buffer_size = std::max(r.max_buffer_size, p.max_buffer_size);
    }
  }
  return r;
}

// KokkosFFT_Distributed_MPI_Extents.hpp:322-417
void check_valid_extents(const Ext& gin, const Ext& gout, const Ext& axes, bool real_input, bool view_layout_right) {
  const std::size_t rank = gin.size();
  if (axes.empty() || axes.size() > rank) fail(kErrInvalidArgument, "input axes are not valid for the view");
  // kokkos-fft are_valid_axes: every axis in range and no duplicates.
  for (std::size_t i = 0; i < axes.size(); ++i) {
    if (axes[i] >= rank) fail(kErrInvalidArgument, "input axes are not valid for the view");
    for (std::size_t j = 0; j < i; ++j)
      if (axes[i] == axes[j]) fail(kErrInvalidArgument, "input axes are not valid for the view");
  }
  Ext map = get_map_axes(rank, axes, view_layout_right);
  Ext in_e = compute_mapped_extents(gin, map), out_e = compute_mapped_extents(gout, map);
  std::size_t inner = view_layout_right ? rank - 1 : 0;
  std::string detail = " in" + ext_str(in_e) + ", out" + ext_str(out_e);
  for (std::size_t i = 0; i < rank; ++i) {
    if (i == inner) continue;
    if (in_e[i] != out_e[i])
      fail(kErrInvalidExtents, "input and output extents must be the same except for the transform axis:" + detail);
  }
  if (!real_input) {
    if (in_e[inner] != out_e[inner])
      fail(kErrInvalidExtents, "input and output extents must be the same for C2C transform:" + detail);
  } else {
    if (out_e[inner] != in_e[inner] / 2 + 1)
      fail(kErrInvalidExtents,
           "For R2C, the 'output extent' of transform must be equal to 'input extent'/2 + 1:" + detail);
  }
}

}  // namespace dfft
