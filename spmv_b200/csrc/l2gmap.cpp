// Host construction of the ghost-map communication pattern for all virtual
// ranks of a communicator at once.
//
// The reference builds the same arrays collectively with MPI (L2GMap.cpp:15-122:
// Allgather of sizes, Alltoall of ghost counts, a symmetric distributed-graph
// communicator, Neighbor_alltoall of counts and Neighbor_alltoallv of the
// requested indices).  With every rank in one process the exchanges are plain
// reads of the other ranks' inputs; the resulting arrays are identical to the
// reference's, member by member, including its quirks:
//  * neighbours are listed in ascending rank order (L2GMap.cpp:64-78);
//  * a rank with no neighbours keeps send_count = recv_count = {0}
//    (L2GMap.cpp:87-92);
//  * send_offset is shifted by local_size (L2GMap.cpp:119-121).
#include <algorithm>
#include <numeric>

#include "internal.h"

namespace spmvb {

namespace {

// Rank owning global index g (ranges is the prefix sum of local sizes).
int owner_of(const std::vector<int64_t>& ranges, int64_t g) {
  auto it = std::upper_bound(ranges.begin(), ranges.end(), g);
  return int(it - ranges.begin()) - 1;
}

}  // namespace

void build_pattern(spmv_l2gmap map, const int64_t* local_size,
                   const int64_t* const* ghosts, const int64_t* num_ghosts) {
  const int P = map->comm->size;
  require(local_size != nullptr, "spmv::L2GMap - Error: local_size is NULL");
  require(num_ghosts != nullptr, "spmv::L2GMap - Error: num_ghosts is NULL");

  map->ranges.assign(P + 1, 0);
  for (int r = 0; r < P; ++r) {
    require(local_size[r] >= 0 && local_size[r] < (int64_t(1) << 31),
            "spmv::L2GMap - Error: local_size out of range");
    require(num_ghosts[r] >= 0 && num_ghosts[r] < (int64_t(1) << 31),
            "spmv::L2GMap - Error: number of ghosts out of range");
    require(num_ghosts[r] == 0 || (ghosts && ghosts[r]),
            "spmv::L2GMap - Error: ghost array is NULL");
    map->ranges[r + 1] = map->ranges[r] + local_size[r];
  }
  const int64_t N = map->ranges[P];

  map->rank.assign(P, RankMap{});
  // counts[r][q]: number of ghosts rank r holds that rank q owns.
  std::vector<std::vector<int32_t>> counts(P, std::vector<int32_t>(P, 0));
  for (int r = 0; r < P; ++r) {
    RankMap& R = map->rank[r];
    R.local_size = local_size[r];
    R.ghosts.assign(ghosts ? ghosts[r] : nullptr,
                    ghosts ? ghosts[r] + num_ghosts[r] : nullptr);
    if (!std::is_sorted(R.ghosts.begin(), R.ghosts.end()))
      fail(SPMV_ERROR_INVALID_ARGUMENT, "Ghosts must be sorted");
    const int64_t r0 = map->ranges[r], r1 = map->ranges[r + 1];
    for (int64_t g : R.ghosts) {
      if (g >= r0 && g < r1)
        fail(SPMV_ERROR_INVALID_ARGUMENT, "Ghost index in local range");
      // The reference asserts (compiled out) that a ghost is a valid global
      // index; an out-of-range ghost would be read out of bounds there.
      require(g >= 0 && g < N,
              "spmv::L2GMap - Error: ghost index outside the global range");
      ++counts[r][owner_of(map->ranges, g)];
    }
  }

  for (int r = 0; r < P; ++r) {
    RankMap& R = map->rank[r];
    // Neighbours: ranks r takes ghosts from, or that take ghosts from r.
    for (int q = 0; q < P; ++q) {
      if (counts[r][q] > 0 || counts[q][r] > 0) {
        R.neighbours.push_back(q);
        R.send_count.push_back(counts[r][q]);
        R.recv_count.push_back(counts[q][r]);
      }
    }
    if (R.neighbours.empty()) {
      R.send_count = {0};
      R.recv_count = {0};
    }
    R.send_offset.assign(1, 0);
    for (int32_t c : R.send_count) R.send_offset.push_back(R.send_offset.back() + c);
    R.recv_offset.assign(1, 0);
    for (int32_t c : R.recv_count) R.recv_offset.push_back(R.recv_offset.back() + c);

    // indexbuf: for each neighbour q (ascending), the owned indices q asked
    // r for, in q's ghost order.  q's ghosts owned by r form one contiguous
    // run of its sorted ghost list.
    R.indexbuf.reserve(R.recv_offset.back());
    for (int q : R.neighbours) {
      const auto& gq = map->rank[q].ghosts;
      auto lo = std::lower_bound(gq.begin(), gq.end(), map->ranges[r]);
      auto hi = std::lower_bound(gq.begin(), gq.end(), map->ranges[r + 1]);
      for (auto it = lo; it != hi; ++it)
        R.indexbuf.push_back(int32_t(*it - map->ranges[r]));
    }
    for (int32_t& s : R.send_offset) s += int32_t(R.local_size);
  }
}

// Device tables for update and reverse_update.
//
// update: ghost slot s of rank q receives owned entry (g - ranges[p]) of the
// owner p of ghost g = ghosts_q[s].
//
// reverse_update: rank r adds databuf[i] into vec_r[indexbuf_r[i]] for i in
// order (L2GMap.cpp:168-169), where databuf_r's segment k holds the ghost
// slots that neighbour q = neighbours_r[k] keeps for r, in q's ghost order.
// Contributions are grouped by target entry, keeping the order of i, so a
// single thread per target repeats the reference's additions exactly.
void build_halo_tables(spmv_l2gmap map) {
  HaloTables& H = map->halo;
  if (H.built) return;
  const int P = map->comm->size;

  std::vector<int32_t> u_ranks, u_dst, u_src;
  for (int q = 0; q < P; ++q) {
    const RankMap& Q = map->rank[q];
    for (size_t s = 0; s < Q.ghosts.size(); ++s) {
      const int64_t g = Q.ghosts[s];
      const int p = owner_of(map->ranges, g);
      u_ranks.push_back((q << 16) | p);
      u_dst.push_back(int32_t(Q.local_size + int64_t(s)));
      u_src.push_back(int32_t(g - map->ranges[p]));
    }
  }

  std::vector<int32_t> t_rank, t_idx, t_ptr{0}, c_rank, c_idx;
  std::vector<int32_t> first_slot(P);  // per rank: start of its ghosts owned by r
  for (int r = 0; r < P; ++r) {
    const RankMap& R = map->rank[r];
    // (target, contributor) pairs in the reference's order.
    std::vector<std::pair<int32_t, std::pair<int32_t, int32_t>>> pairs;
    pairs.reserve(R.indexbuf.size());
    size_t i = 0;
    for (size_t k = 0; k < R.neighbours.size(); ++k) {
      const int q = R.neighbours[k];
      const auto& gq = map->rank[q].ghosts;
      const int64_t slot0 =
          std::lower_bound(gq.begin(), gq.end(), map->ranges[r]) - gq.begin();
      for (int32_t j = 0; j < R.recv_count[k]; ++j, ++i) {
        const int32_t src = int32_t(map->rank[q].local_size + slot0 + j);
        pairs.push_back({R.indexbuf[i], {q, src}});
      }
    }
    // Stable sort by target keeps the order of i within each target.
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t a = 0; a < pairs.size();) {
      size_t b = a;
      while (b < pairs.size() && pairs[b].first == pairs[a].first) {
        c_rank.push_back(pairs[b].second.first);
        c_idx.push_back(pairs[b].second.second);
        ++b;
      }
      t_rank.push_back(r);
      t_idx.push_back(pairs[a].first);
      t_ptr.push_back(int32_t(c_rank.size()));
      a = b;
    }
  }

  auto up = [](DevBuf& buf, const std::vector<int32_t>& v) {
    buf.reserve(std::max<size_t>(v.size(), 1) * sizeof(int32_t));
    if (!v.empty())
      SPMVB_CUDA(cudaMemcpy(buf.ptr, v.data(), v.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice));
  };
  DeviceGuard dg(map->comm->device);
  up(H.upd_ranks, u_ranks);
  up(H.upd_dst, u_dst);
  up(H.upd_src, u_src);
  up(H.rev_tgt_rank, t_rank);
  up(H.rev_tgt_idx, t_idx);
  up(H.rev_ptr, t_ptr);
  up(H.rev_src_rank, c_rank);
  up(H.rev_src_idx, c_idx);
  H.n_update = int64_t(u_dst.size());
  H.n_targets = int64_t(t_idx.size());
  H.n_contrib = int64_t(c_idx.size());
  H.built = true;
}

}  // namespace spmvb
