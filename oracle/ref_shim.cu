// Test-only accessor shim for the reference solver (oracle/_ref build only).
//
// This translation unit is compiled by oracle/Makefile together with the
// reference's native/xpbd_capi.cu into oracle/_ref/libxpbd_ref.so.  It pulls in
// the reference solver translation unit (native/solver_core/cuda_rasterizer/
// forward.cu) with #include, straight from the reference checkout named on the
// compiler's include path, so that the parity tests can read the solver's
// file-static stage buffers (hash keys, sorted order, candidate lists, cluster
// CSR, colourings) and flip the Gauss-Seidel toggles that the reference C ABI
// does not export.  Nothing here is shipped; the product library never links it.
//
// Every accessor copies device data to a caller-owned host buffer and returns the
// element count (or -1 when the buffer does not exist or is too small).
#include "forward.cu"

namespace {
template <typename T>
int copy_out(const T* dev, long long count, T* host, long long cap)
{
	if (!dev || count < 0) return -1;
	if (!host) return (int)count;
	if (cap < count) return -1;
	if (count > 0) cudaMemcpy(host, dev, sizeof(T) * (size_t)count, cudaMemcpyDeviceToHost);
	return (int)count;
}
}  // namespace

extern "C" {

// Gauss-Seidel toggles (forward.cu:3780-3812; not reachable through xpbd_capi.cu).
__attribute__((visibility("default"))) void refshim_set_gs(int distance, int volume)
{
	FORWARD::setDistanceGSEnabled(distance != 0);
	FORWARD::setVolumeGSEnabled(volume != 0);
}

// Volume Kernel A/B execution shape (forward.cu:4043-4060): 0 auto, 1 thread, 2 warp.
__attribute__((visibility("default"))) void refshim_set_volume_warp_mode(int mode)
{
	FORWARD::setVolumeWarpMode(mode);
}

// Sizes: [0] N, [1] directed CSR length, [2] volume member total, [3] reverse total,
// [4] GS edges, [5] GS edge colours, [6] volume GS clusters, [7] volume GS colours,
// [8] self-collision table size, [9] self-collision candidates last step.
__attribute__((visibility("default"))) void refshim_sizes(long long* out)
{
	const int N = cm_num_elements;
	long long volTotal = 0, revTotal = 0;
	if (N > 0 && d_volCount) {
		std::vector<int> c(N);
		cudaMemcpy(c.data(), d_volCount, sizeof(int) * N, cudaMemcpyDeviceToHost);
		for (int v : c) volTotal += v;
	}
	if (N > 0 && d_volRevCount) {
		std::vector<int> c(N);
		cudaMemcpy(c.data(), d_volRevCount, sizeof(int) * N, cudaMemcpyDeviceToHost);
		for (int v : c) revTotal += v;
	}
	out[0] = N;
	out[1] = cm_num_neighbors;
	out[2] = volTotal;
	out[3] = revTotal;
	out[4] = g_gsNumEdges;
	out[5] = g_gsColorOffset.empty() ? 0 : (long long)g_gsColorOffset.size() - 1;
	out[6] = g_volGSColorOffset.empty() ? 0 : g_volGSColorOffset.back();
	out[7] = g_volGSColorOffset.empty() ? 0 : (long long)g_volGSColorOffset.size() - 1;
	out[8] = g_selfColTable;
	out[9] = g_selfColContacts;
}

// Runs the reference's once-per-step self-collision build (forward.cu:11796-11849) on
// caller-given start positions x[3N] and predicted positions p[3N], exactly as a step
// would after predict.  Needs the graph on the device (one xpbd_step first).
// Returns the candidate total, or -1.
__attribute__((visibility("default"))) int refshim_selfcol_build(const float* x, const float* p)
{
	const int N = cm_num_elements;
	if (N <= 0 || !d_pos_curr || !d_pos_next || !x || !p) return -1;
	cudaMemcpy(d_pos_curr, x, sizeof(float3) * N, cudaMemcpyHostToDevice);
	cudaMemcpy(d_pos_next, p, sizeof(float3) * N, cudaMemcpyHostToDevice);
	const int threads = 256;
	selfColBuild(N, (N + threads - 1) / threads, threads);
	cudaDeviceSynchronize();
	return g_selfColContacts;
}

__attribute__((visibility("default"))) int refshim_int(const char* name, int* out, long long cap)
{
	const int N = cm_num_elements;
	const std::string s(name);
	long long sz[10];
	refshim_sizes(sz);
	if (s == "vol_offset") return copy_out(d_volOffset, N, out, cap);
	if (s == "vol_count") return copy_out(d_volCount, N, out, cap);
	if (s == "vol_idx") return copy_out(d_volIdx, sz[2], out, cap);
	if (s == "rev_offset") return copy_out(d_volRevOffset, N, out, cap);
	if (s == "rev_count") return copy_out(d_volRevCount, N, out, cap);
	if (s == "rev_idx") return copy_out(d_volRevIdx, sz[3], out, cap);
	if (s == "mat_type") return copy_out(d_matType, N, out, cap);
	if (s == "nbr_offset") return copy_out(d_offset, N, out, cap);
	if (s == "nbr_count") return copy_out(d_nbrCount, N, out, cap);
	if (s == "nbr_idx") return copy_out(d_nbrIdx, sz[1], out, cap);
	if (s == "gs_edge") return copy_out(reinterpret_cast<const int*>(d_gsEdge), 2 * sz[4], out, cap);
	if (s == "gs_color_offset") {
		const long long n = (long long)g_gsColorOffset.size();
		if (!out) return (int)n;
		if (cap < n) return -1;
		for (long long i = 0; i < n; ++i) out[i] = g_gsColorOffset[(size_t)i];
		return (int)n;
	}
	if (s == "vol_gs_order") return copy_out(d_volGSOrder, sz[6], out, cap);
	if (s == "vol_gs_color_offset") {
		const long long n = (long long)g_volGSColorOffset.size();
		if (!out) return (int)n;
		if (cap < n) return -1;
		for (long long i = 0; i < n; ++i) out[i] = g_volGSColorOffset[(size_t)i];
		return (int)n;
	}
	if (s == "sc_keys") return copy_out(reinterpret_cast<const int*>(d_scKeys), N, out, cap);
	if (s == "sc_keys_sorted") return copy_out(reinterpret_cast<const int*>(d_scKeysSorted), N, out, cap);
	if (s == "sc_idx_sorted") return copy_out(d_scIdxSorted, N, out, cap);
	if (s == "sc_cell_start") return copy_out(d_scCellStart, g_selfColTable, out, cap);
	if (s == "sc_cell_end") return copy_out(d_scCellEnd, g_selfColTable, out, cap);
	if (s == "sc_contact") return copy_out(d_scContact, (long long)N * SELFCOL_MAX_CONTACTS, out, cap);
	if (s == "sc_count") return copy_out(d_scCount, N, out, cap);
	if (s == "obj_id") return copy_out(d_objId, N, out, cap);
	return -1;
}

__attribute__((visibility("default"))) int refshim_float(const char* name, float* out, long long cap)
{
	const int N = cm_num_elements;
	const std::string s(name);
	long long sz[10];
	refshim_sizes(sz);
	if (s == "det_rest") return copy_out(d_detSigmaRest, N, out, cap);
	if (s == "sigma_rest") return copy_out(d_Sigma_rest, 6LL * N, out, cap);
	if (s == "v_rest") return copy_out(d_V_rest, N, out, cap);
	if (s == "rest_len") return copy_out(d_volRestLen, N, out, cap);
	if (s == "gs_rest") return copy_out(d_gsRest, sz[4], out, cap);
	if (s == "gs_stiff") return copy_out(d_gsStiff, sz[4], out, cap);
	if (s == "vel") return copy_out(reinterpret_cast<const float*>(d_vel), 3LL * N, out, cap);
	if (s == "pos_rest") return copy_out(reinterpret_cast<const float*>(d_pos_rest), 3LL * N, out, cap);
	if (s == "pos_next") return copy_out(reinterpret_cast<const float*>(d_pos_next), 3LL * N, out, cap);
	if (s == "inv_mass") return copy_out(d_invMass, N, out, cap);
	if (s == "cluster_coef") return copy_out(d_volClusterCoef, N, out, cap);
	if (s == "cm_time") return copy_out(d_time_curr, N, out, cap);
	if (s == "self_col") {
		// [0] spacing, [1] contact distance d_c, [2] cell size (reach)
		if (!out) return 3;
		if (cap < 3) return -1;
		out[0] = g_selfColSpacing;
		out[1] = g_selfColRadiusScale * g_selfColSpacing;
		out[2] = g_selfColReach;
		return 3;
	}
	return -1;
}

// ChainMail (forward.cu:12808-13006): not reachable through xpbd_capi.cu, which forces
// XPBD mode (xpbd_capi.cu:98).  These drive the reference's own seed kernel and its
// runChainmailGPU on the graph a first xpbd_step uploaded.
__attribute__((visibility("default"))) void refshim_chainmail_set_material(float global_scale, float air, float skin,
	float bone, int use_edge_stiffness, float edge_influence)
{
	FORWARD::setChainmailMaterialParams(global_scale, air, skin, bone, use_edge_stiffness != 0, edge_influence);
}

// applySeedCommandsKernel (forward.cu:5907-5924): seeds move by delta, arrival time 0.
__attribute__((visibility("default"))) int refshim_chainmail_seed(int count, const int* idx, const float* delta)
{
	const int N = cm_num_elements;
	if (N <= 0 || !d_pos_curr || !d_time_curr || count < 0) return -1;
	if (count == 0) return 0;
	int* di = nullptr;
	float3* dd = nullptr;
	cudaMalloc(&di, sizeof(int) * count);
	cudaMalloc(&dd, sizeof(float3) * count);
	cudaMemcpy(di, idx, sizeof(int) * count, cudaMemcpyHostToDevice);
	cudaMemcpy(dd, delta, sizeof(float3) * count, cudaMemcpyHostToDevice);
	applySeedCommandsKernel<<<(count + 255) / 256, 256>>>(count, di, dd, d_pos_curr, d_time_curr, (int*)nullptr);
	cudaDeviceSynchronize();
	cudaFree(di);
	cudaFree(dd);
	return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// runChainmailGPU's dense path (no active map, no inertia: the reference defaults,
// forward.cu:47 and 73).  Its ChainMail argument only supplies the element count here
// (no host upload or download), so a placeholder with N elements is passed.
__attribute__((visibility("default"))) int refshim_chainmail_run(int prop_iters, int relax_iters, float prop_strength,
	float relax_stiffness, float relax_damping)
{
	const int N = cm_num_elements;
	if (N <= 0 || !d_pos_curr || !d_time_curr) return -1;
	static FORWARD::ChainMail placeholder;
	if ((int)placeholder.numElements() != N)
		placeholder.loadGraph(placeholder, std::vector<FORWARD::Pos>(N, FORWARD::Pos(0.0f)), std::vector<FORWARD::Edge>(),
			std::vector<float>(N, 0.0f));
	g_useActiveMap = false;
	g_cmInertiaGain = 0.0f;
	runChainmailGPU(placeholder, prop_iters, relax_iters, prop_strength, relax_stiffness, relax_damping, false, false,
		nullptr);
	cudaDeviceSynchronize();
	return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // extern "C"
