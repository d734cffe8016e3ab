// Internal declarations of the B200 XPBD engine (not part of the public C ABI).
//
// Device layout (one scene, N Gaussians, M directed graph edges):
//   pos_curr / pos_next / pos_tmp   float4[N]  xyz + inverse mass in w (128-bit loads)
//   vel                             float4[N]  xyz, w unused
//   pos_rest                        float4[N]  xyz + 0
//   pos_out                         float3[N]  committed positions in the caller's float3
//                                              layout (xpbd_positions_device)
//   off                             int[N+1]   graph CSR row starts (both edge directions)
//   nbr / ndist / nstiff / lam      [M]        neighbour index, rest length, stiffness,
//                                              distance multiplier (updated in place)
//   vol_off / vol_idx               cluster members (leader excluded), CSR over leaders
//   rev_off / rev_idx               clusters containing each node (transposed CSR)
//   rec                             float4[3N] cluster blackboard, 36 B used per cluster:
//                                              float4[2N] (M xx, yy, zz, xy), (M xz, yz, c.x, c.y)
//                                              with M = coef Sinv, then float[N] c.z; c.x = NaN: no record
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace xpbd {

constexpr int kMaxColliders = 32;   // forward.cu:128
constexpr int kColliderAcc = 7;     // forward.cu:145
constexpr int kSelfColMax = 32;     // forward.cu:223
constexpr int kBlock = 256;

struct KinCollider {                // forward.cu:129-136
	float R[9];
	float t[3];
	float h[3];
	int type;
	float Rp[9];
	float tp[3];
	int obj;                        // object it acts on, -1 every Gaussian (batched scenes)
};

// Step parameters read by every kernel from device memory, so that one captured
// CUDA graph serves every step even when settings or collider poses change.
struct StepParams {
	float dt;
	float inv_mass_scale;
	float stiffness_scale;
	float under_relax;
	float dist_compliance;
	float vol_compliance;
	float shape_compliance;
	float shape_blend;
	float vel_damping;
	float gx, gy, gz;               // gravity (predict)
	int ground_on;
	float gn[3];                    // ground normal
	float ground_plane;             // height + contact radius
	float ground_slop, ground_friction, ground_restitution, resting_speed;
	int kin_count;
	float kin_margin, kin_friction;
	float sc_dc, sc_search, sc_excl2, sc_cross_excl2, sc_fast_rel, sc_search_plus16dc;
	int sc_within;
	int sc_single_object;           // every particle has the same object id
	int kin_filtered;               // some collider acts on one object only
	int kin_ext_ranges;             // objects with a range in the batched collider list
	int press_on, press_axis;       // press harness plates on the rest axis (forward.cu:9411-9424)
	float press_lo, press_hi;
	KinCollider kin[kMaxColliders];
};

// Counters written by kernels, read back on demand.
struct DevCounters {
	unsigned int sc_contacts;       // candidate total (forward.cu:6984 [0])
	unsigned int sc_overflow;       // over-cap replacements ([1])
	unsigned int sc_max_disp2_bits; // max predict displacement^2 (float bits, >= 0)
	float sc_inv_cell;              // 1 / cell size
	float sc_reach;
	unsigned int shapes_deformed;
	unsigned int shapes_kept;
	unsigned int sc_active;         // Gaussians in the grid when the object box filter is on ([2])
	unsigned int bar_count, bar_gen; // grid barrier of the fused substep launch
	unsigned int bar_timeout;       // a barrier wait of the fused launch ran out (error)
	// near-pair grid of one-object scenes: box of the predicted positions (order-preserving
	// images; the minimum complemented), origin, 1 / cell and cells per axis
	unsigned int nb_lo[3], nb_hi[3];
	float nb_origin[3], nb_inv;
	int nb_dim[3];
	int kin_hits[kMaxColliders];
	float kin_push[kMaxColliders * kColliderAcc];
	double jstats[3];               // sum V, sum V J, sum V J^2
};

// Host-side graph data produced at upload (builder.cpp).
struct HostGraph {
	int n = 0;
	std::vector<int> off;           // N+1
	std::vector<int> nbr;
	std::vector<float> ndist, nstiff;
};

struct HostClusters {
	std::vector<int> vol_off;       // N+1
	std::vector<int> vol_idx;
	std::vector<int> rev_off;       // N+1
	std::vector<int> rev_idx;
	int leaders = 0;
	float avg_members = 0.0f;
	std::vector<int> gs_order;      // leaders in colour order
	std::vector<int> gs_color_off;  // colours + 1
	int gs_lower_bound = 0;
};

struct HostEdgeColoring {
	std::vector<int2> edge;
	std::vector<float> rest, stiff;
	std::vector<int> color_off;
};

// builder.cpp
void build_graph(int n, int e, const int* edges, const float* rest, const float* stiff, HostGraph& g);
void build_clusters(const HostGraph& g, const float* rest_pos3, int ring_k, int cap, int leader_min_hop,
	HostClusters& out);
// the same from every node's member list built on the GPU: node i's list at
// lidx[loff[i] ...], counts[i] entries, or counts[i] = -1 where the host builds it
void build_clusters_from_lists(const HostGraph& g, const float* rest_pos3, int ring_k, int cap, int leader_min_hop,
	const std::vector<long long>& loff, const std::vector<int>& lidx, const std::vector<int>& counts,
	HostClusters& out);
void build_edge_coloring(const HostGraph& g, HostEdgeColoring& out);
void build_components(const HostGraph& g, int min_component, std::vector<int>& obj_id, int& num_objects);
float graph_spacing(const HostGraph& g);

}  // namespace xpbd
