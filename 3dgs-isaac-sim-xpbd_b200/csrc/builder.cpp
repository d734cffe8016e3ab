// Upload-time graph builders (host C++, std::thread).
//
// These produce the integer topology the solver kernels consume.  They follow the
// reference's construction steps exactly, because the cluster membership, the
// transposed membership and both colourings are part of the parity contract
// (bit-exact with the reference):
//   build_graph         ChainMail::loadGraph            forward.cu:2702-2779
//   build_clusters      rebuildVolumeClusters           forward.cu:9814-10246
//                       (k-hop BFS, HARD_CAP 8192, farthest-point subsample,
//                        r>=2 greedy cover, transposed CSR with leader self entries)
//                       + buildVolumeGSColors           forward.cu:9745-9812
//   build_edge_coloring buildDistanceGSEdges            forward.cu:10407-10517
//   build_components    objectEnsureComponents          forward.cu:11309-11374
//   graph_spacing       selfColEnsureSpacing            forward.cu:11761-11792
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "xpbd_internal.h"

namespace xpbd {

void build_graph(int n, int e, const int* edges, const float* rest, const float* stiff, HostGraph& g)
{
	g.n = n;
	std::vector<int> cnt(n, 0);
	for (int k = 0; k < e; ++k) {
		const int a = edges[2 * k], b = edges[2 * k + 1];
		if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
		++cnt[a];
		++cnt[b];
	}
	g.off.assign(n + 1, 0);
	for (int i = 0; i < n; ++i) g.off[i + 1] = g.off[i] + cnt[i];
	const int m = g.off[n];
	g.nbr.resize(m);
	g.ndist.resize(m);
	g.nstiff.resize(m);
	std::vector<int> fill(g.off.begin(), g.off.end() - 1);
	// each undirected edge lands in both endpoint lists, in input order
	for (int k = 0; k < e; ++k) {
		const int a = edges[2 * k], b = edges[2 * k + 1];
		if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
		const int ea = fill[a]++, eb = fill[b]++;
		g.nbr[ea] = b; g.ndist[ea] = rest[k]; g.nstiff[ea] = stiff[k];
		g.nbr[eb] = a; g.ndist[eb] = rest[k]; g.nstiff[eb] = stiff[k];
	}
}

namespace {

constexpr int kHardCap = 8192;

struct Scratch {
	std::vector<int> stamp, frontier, next, collected;
	std::vector<float> md;
	std::vector<char> taken;
	explicit Scratch(int n) : stamp(n, -1) {}
};

inline float dist2(const float* a, const float* b)
{
	const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
	return dx * dx + dy * dy + dz * dz;
}

// k-hop BFS from leader i, then farthest-point subsample to `cap` members.
void members_of(const HostGraph& g, const float* rest, int i, int k, int cap, Scratch& s, std::vector<int>& out)
{
	const int n = g.n;
	auto& col = s.collected;
	col.clear();
	if (k <= 1) {
		for (int e = g.off[i]; e < g.off[i + 1]; ++e) {
			const int j = g.nbr[e];
			if (j >= 0 && j < n && j != i) col.push_back(j);
		}
	}
	else {
		s.frontier.clear();
		s.stamp[i] = i;
		s.frontier.push_back(i);
		for (int d = 0; d < k && !s.frontier.empty() && (int)col.size() < kHardCap; ++d) {
			s.next.clear();
			bool capped = false;
			for (int f : s.frontier) {
				for (int e = g.off[f]; e < g.off[f + 1]; ++e) {
					const int j = g.nbr[e];
					if (j < 0 || j >= n || s.stamp[j] == i) continue;
					s.stamp[j] = i;
					col.push_back(j);
					s.next.push_back(j);
					if ((int)col.size() >= kHardCap) { capped = true; break; }
				}
				if (capped) break;
			}
			s.frontier.swap(s.next);
			if (capped) break;
		}
	}
	out.clear();
	if ((int)col.size() <= cap) {
		out.assign(col.begin(), col.end());
		return;
	}
	// farthest point: start at the candidate farthest from the leader; every pick
	// lowers the remaining candidates' distance-to-picked; next = first maximum
	const int mc = (int)col.size();
	s.md.resize(mc);
	s.taken.assign(mc, 0);
	const float* cpos = rest + 3 * (size_t)i;
	int cur = 0;
	float best = -1.0f;
	for (int m = 0; m < mc; ++m) {
		const float dd = dist2(rest + 3 * (size_t)col[m], cpos);
		s.md[m] = dd;
		if (dd > best) { best = dd; cur = m; }
	}
	out.reserve(cap);
	for (int t = 0; t < cap; ++t) {
		s.taken[cur] = 1;
		out.push_back(col[cur]);
		const float* cp = rest + 3 * (size_t)col[cur];
		int nxt = -1;
		float nbest = -1.0f;
		for (int m = 0; m < mc; ++m) {
			if (s.taken[m]) continue;
			const float dd = dist2(rest + 3 * (size_t)col[m], cp);
			if (dd < s.md[m]) s.md[m] = dd;
			if (s.md[m] > nbest) { nbest = s.md[m]; nxt = m; }
		}
		if (nxt < 0) break;
		cur = nxt;
	}
}

// members_of_leader(l) -> (pointer, count) of leader l's member list
template <typename Members>
void color_clusters(int n, const Members& members_of_leader, const std::vector<char>& leader, HostClusters& out)
{
	out.gs_order.clear();
	out.gs_color_off.clear();
	out.gs_lower_bound = 0;
	double work = 0.0;
	for (int j = 0; j < n; ++j) {
		const int h = out.rev_off[j + 1] - out.rev_off[j];
		out.gs_lower_bound = std::max(out.gs_lower_bound, h);
		work += (double)h * h;
	}
	int m = 0;
	for (int i = 0; i < n; ++i) m += leader[i] ? 1 : 0;
	if (m == 0 || work > 4.0e9) return;
	std::vector<int> color(n, -1), stamp;
	int num_colors = 0;
	for (int l = 0; l < n; ++l) {
		if (!leader[l]) continue;
		if ((int)stamp.size() < num_colors + 1) stamp.resize(num_colors + 1, -1);
		auto forbid = [&](int j) {
			for (int q = out.rev_off[j]; q < out.rev_off[j + 1]; ++q) {
				const int c = out.rev_idx[q];
				if (c >= 0 && c < n && color[c] >= 0) stamp[color[c]] = l;
			}
		};
		forbid(l);
		const auto ml = members_of_leader(l);
		for (int t = 0; t < ml.second; ++t) {
			const int j = ml.first[t];
			if (j >= 0 && j < n) forbid(j);
		}
		int c = 0;
		while (c < num_colors && stamp[c] == l) ++c;
		color[l] = c;
		num_colors = std::max(num_colors, c + 1);
	}
	out.gs_color_off.assign(num_colors + 1, 0);
	for (int l = 0; l < n; ++l)
		if (leader[l]) out.gs_color_off[color[l] + 1]++;
	for (int c = 0; c < num_colors; ++c) out.gs_color_off[c + 1] += out.gs_color_off[c];
	std::vector<int> fill(out.gs_color_off.begin(), out.gs_color_off.end() - 1);
	out.gs_order.resize(m);
	for (int l = 0; l < n; ++l)
		if (leader[l]) out.gs_order[fill[color[l]]++] = l;
}

// Member CSR, transposed membership (leader self entry first, then clusters in leader
// order) and the cluster colouring, from the leaders' member lists.
template <typename Members>
void finish_clusters(int n, const Members& members_of_leader, const std::vector<char>& leader, HostClusters& out)
{
	out.vol_off.assign(n + 1, 0);
	for (int i = 0; i < n; ++i) out.vol_off[i + 1] = out.vol_off[i] + members_of_leader(i).second;
	out.vol_idx.resize(std::max(out.vol_off[n], 1));
	for (int i = 0; i < n; ++i) {
		const auto mi = members_of_leader(i);
		std::copy(mi.first, mi.first + mi.second, out.vol_idx.begin() + out.vol_off[i]);
	}
	std::vector<int> rc(n, 0);
	for (int i = 0; i < n; ++i) rc[i] += leader[i] ? 1 : 0;
	for (int i = 0; i < n; ++i) {
		const auto mi = members_of_leader(i);
		for (int t = 0; t < mi.second; ++t) ++rc[mi.first[t]];
	}
	out.rev_off.assign(n + 1, 0);
	for (int i = 0; i < n; ++i) out.rev_off[i + 1] = out.rev_off[i] + rc[i];
	out.rev_idx.resize(std::max(out.rev_off[n], 1));
	std::vector<int> cur(out.rev_off.begin(), out.rev_off.end() - 1);
	for (int i = 0; i < n; ++i)
		if (leader[i]) out.rev_idx[cur[i]++] = i;
	for (int i = 0; i < n; ++i) {
		const auto mi = members_of_leader(i);
		for (int t = 0; t < mi.second; ++t) out.rev_idx[cur[mi.first[t]]++] = i;
	}
	out.avg_members = out.leaders > 0 ? (float)((double)out.vol_off[n] / out.leaders) : 0.0f;
	color_clusters(n, members_of_leader, leader, out);
}

}  // namespace

namespace {

// Leader selection of rebuildVolumeClusters for leader spacing r >= 2 (forward.cu:
// 10070-10132): in index order, a node whose cover is below the target (min(r, 6)) and
// that no earlier leader suppressed (within r - 1 hops) becomes a leader, and its list
// raises the cover of itself and its members; then under-covered nodes are promoted
// until none is left.  list_of(i) -> (pointer, count) of node i's member list, the same
// whoever asks (the reference's cover cap is 0, so a list depends on the node alone).
template <typename ListOf>
int cover_leaders(const HostGraph& g, int leader_r, const ListOf& list_of, std::vector<char>& leader)
{
	const int n = g.n;
	const int target = std::max(1, std::min(6, leader_r));
	std::vector<int> cover(n, 0), stamp_r(n, -1);
	int count = 0;
	std::vector<int> fr, nx;
	auto take = [&](int i) {
		leader[i] = 1;
		++count;
		const auto m = list_of(i);
		++cover[i];
		for (int t = 0; t < m.second; ++t) {
			const int j = m.first[t];
			if (j >= 0 && j < n) ++cover[j];
		}
	};
	for (int seed = 0; seed < n; ++seed) {
		if (cover[seed] >= target) continue;
		if (stamp_r[seed] == -2) continue;
		take(seed);
		fr.clear();
		stamp_r[seed] = -2;
		fr.push_back(seed);
		for (int d = 0; d < leader_r - 1 && !fr.empty(); ++d) {
			nx.clear();
			for (int f : fr)
				for (int e = g.off[f]; e < g.off[f + 1]; ++e) {
					const int j = g.nbr[e];
					if (j < 0 || j >= n || stamp_r[j] == -2) continue;
					stamp_r[j] = -2;
					nx.push_back(j);
				}
			fr.swap(nx);
		}
	}
	bool progressed = true;
	while (progressed) {
		progressed = false;
		for (int i = 0; i < n; ++i) {
			if (cover[i] >= target || leader[i]) continue;
			take(i);
			progressed = true;
		}
	}
	return count;
}

}  // namespace

void build_clusters_from_lists(const HostGraph& g, const float* rest, int ring_k, int cap, int leader_min_hop,
	const std::vector<long long>& loff, const std::vector<int>& lidx, const std::vector<int>& counts,
	HostClusters& out)
{
	// every node's list from the GPU (loff / lidx), or -1 in counts where the host builds it
	const int n = g.n;
	const int leader_r = std::max(1, leader_min_hop);
	std::vector<std::vector<int>> host_lists;
	std::vector<int> host_at(n, -1);
	Scratch sc(n);
	auto list_of = [&](int i) -> std::pair<const int*, int> {
		if (counts[i] >= 0) return std::make_pair(lidx.data() + loff[i], counts[i]);
		if (host_at[i] < 0) {
			host_at[i] = (int)host_lists.size();
			host_lists.emplace_back();
			members_of(g, rest, i, ring_k, cap, sc, host_lists.back());
		}
		const auto& v = host_lists[host_at[i]];
		return std::make_pair((const int*)v.data(), (int)v.size());
	};
	std::vector<char> leader(n, 0);
	if (leader_r <= 1) {
		std::fill(leader.begin(), leader.end(), (char)1);
		out.leaders = n;
		for (int i = 0; i < n; ++i)
			if (counts[i] < 0) list_of(i);   // build the host lists before the parallel reads
	}
	else
		out.leaders = cover_leaders(g, leader_r, list_of, leader);
	finish_clusters(n, [&](int i) {
		if (!leader[i]) return std::make_pair((const int*)nullptr, 0);
		return list_of(i);
	}, leader, out);
}

void build_clusters(const HostGraph& g, const float* rest, int ring_k, int cap, int leader_min_hop, HostClusters& out)
{
	const int n = g.n;
	const int leader_r = std::max(1, leader_min_hop);
	std::vector<char> leader(n, 0);
	std::vector<std::vector<int>> members(n);
	if (leader_r <= 1) {
		std::fill(leader.begin(), leader.end(), (char)1);
		out.leaders = n;
		const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
		std::atomic<int> next{ 0 };
		const int chunk = 512;
		auto worker = [&]() {
			Scratch s(n);
			for (;;) {
				const int start = next.fetch_add(chunk);
				if (start >= n) break;
				const int end = std::min(n, start + chunk);
				for (int i = start; i < end; ++i) members_of(g, rest, i, ring_k, cap, s, members[i]);
			}
		};
		std::vector<std::thread> pool;
		for (unsigned t = 0; t < hw; ++t) pool.emplace_back(worker);
		for (auto& th : pool) th.join();
	}
	else {
		// greedy cover, each leader's list built when it is chosen
		Scratch s(n);
		out.leaders = cover_leaders(g, leader_r, [&](int i) {
			if (members[i].empty()) members_of(g, rest, i, ring_k, cap, s, members[i]);
			return std::make_pair((const int*)members[i].data(), (int)members[i].size());
		}, leader);
	}
	finish_clusters(n, [&](int i) {
		if (!leader[i]) return std::make_pair((const int*)nullptr, 0);
		return std::make_pair((const int*)members[i].data(), (int)members[i].size());
	}, leader, out);
}

void build_edge_coloring(const HostGraph& g, HostEdgeColoring& out)
{
	const int n = g.n;
	out.edge.clear();
	out.rest.clear();
	out.stiff.clear();
	out.color_off.clear();
	struct E { int a, b; float rest, stiff; int dup; };
	std::vector<E> dir;
	dir.reserve(g.nbr.size());
	for (int i = 0; i < n; ++i)
		for (int e = g.off[i]; e < g.off[i + 1]; ++e) {
			const int j = g.nbr[e];
			if (j < 0 || j >= n || j == i) continue;
			dir.push_back({ std::min(i, j), std::max(i, j), g.ndist[e], g.nstiff[e], 1 });
		}
	std::sort(dir.begin(), dir.end(), [](const E& x, const E& y) { return x.a != y.a ? x.a < y.a : x.b < y.b; });
	std::vector<E> und;
	und.reserve(dir.size());
	for (const E& x : dir) {
		if (!und.empty() && und.back().a == x.a && und.back().b == x.b) {
			und.back().rest += x.rest;
			und.back().stiff += x.stiff;
			und.back().dup++;
		}
		else und.push_back(x);
	}
	for (E& x : und) {
		x.rest /= float(x.dup);
		x.stiff /= float(x.dup);
	}
	const int ne = (int)und.size();
	if (ne == 0) return;
	std::vector<int> deg(n, 0);
	for (const E& x : und) { deg[x.a]++; deg[x.b]++; }
	const int max_deg = *std::max_element(deg.begin(), deg.end());
	const int words = (2 * max_deg + 63) / 64;
	std::vector<unsigned long long> used((size_t)n * words, 0ull);
	std::vector<int> color(ne);
	int num_colors = 0;
	for (int e = 0; e < ne; ++e) {
		unsigned long long* ua = &used[(size_t)und[e].a * words];
		unsigned long long* ub = &used[(size_t)und[e].b * words];
		int c = -1;
		for (int w = 0; w < words && c < 0; ++w) {
			const unsigned long long free_bits = ~(ua[w] | ub[w]);
			if (!free_bits) continue;
			c = w * 64 + __builtin_ctzll(free_bits);   // lowest free colour
		}
		ua[c >> 6] |= 1ull << (c & 63);
		ub[c >> 6] |= 1ull << (c & 63);
		color[e] = c;
		num_colors = std::max(num_colors, c + 1);
	}
	out.color_off.assign(num_colors + 1, 0);
	for (int e = 0; e < ne; ++e) out.color_off[color[e] + 1]++;
	for (int c = 0; c < num_colors; ++c) out.color_off[c + 1] += out.color_off[c];
	std::vector<int> fill(out.color_off.begin(), out.color_off.end() - 1);
	out.edge.resize(ne);
	out.rest.resize(ne);
	out.stiff.resize(ne);
	for (int e = 0; e < ne; ++e) {
		const int p = fill[color[e]]++;
		out.edge[p] = make_int2(und[e].a, und[e].b);
		out.rest[p] = und[e].rest;
		out.stiff[p] = und[e].stiff;
	}
}

static int find_root(std::vector<int>& parent, int x)
{
	while (parent[x] != x) {
		parent[x] = parent[parent[x]];
		x = parent[x];
	}
	return x;
}

void build_components(const HostGraph& g, int min_component, std::vector<int>& obj_id, int& num_objects)
{
	const int n = g.n;
	std::vector<int> parent(n);
	for (int i = 0; i < n; ++i) parent[i] = i;
	for (int i = 0; i < n; ++i)
		for (int e = g.off[i]; e < g.off[i + 1]; ++e) {
			const int j = g.nbr[e];
			if (j < 0 || j >= n) continue;
			const int ri = find_root(parent, i), rj = find_root(parent, j);
			if (ri != rj) parent[ri] = rj;
		}
	std::vector<int> size(n, 0);
	for (int i = 0; i < n; ++i) ++size[find_root(parent, i)];
	std::vector<int> root_id(n, -1);
	obj_id.assign(n, -1);
	int k = 0;
	for (int i = 0; i < n; ++i) {
		const int r = find_root(parent, i);
		if (root_id[r] == -1) root_id[r] = (size[r] >= min_component) ? k++ : -2;
		if (root_id[r] >= 0) obj_id[i] = root_id[r];
	}
	num_objects = k;
}

float graph_spacing(const HostGraph& g)
{
	std::vector<float> mins;
	mins.reserve(g.n);
	for (int i = 0; i < g.n; ++i) {
		float m = FLT_MAX;
		for (int e = g.off[i]; e < g.off[i + 1]; ++e) {
			const float d = g.ndist[e];
			if (d > 0.0f && std::isfinite(d) && d < m) m = d;
		}
		if (m < FLT_MAX) mins.push_back(m);
	}
	if (mins.empty()) return 0.0f;
	std::nth_element(mins.begin(), mins.begin() + mins.size() / 2, mins.end());
	return mins[mins.size() / 2];
}

}  // namespace xpbd
