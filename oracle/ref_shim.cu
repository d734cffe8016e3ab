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

#include <cub/device/device_scan.cuh>

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


// ---- the viewer's rasteriser on explicit inputs ----
// The reference's own preprocessCUDA (forward.cu:1919-2467; demo modes off, no
// neighbour graph, so the given shapes are used as they are) and renderCUDA
// (forward.cu:2469-2650, through FORWARD::render), with the binning steps of
// Rasterizer::forward (rasterizer_impl.cu:330-370: inclusive scan of touched tiles,
// pair keys tile << 32 | depth written in Gaussian order, cub stable radix sort over
// 32 + bits(tiles) bits, tile ranges) done by the small kernels below.
namespace refrender {

// the reference's bit count of the tile id (getHigherMsb, rasterizer_impl.cu:34-49 is
// file-local there): the smallest b with n >> b == 0
int getHigherMsb(uint32_t n)
{
	int b = 0;
	while (b < 32 && (n >> b)) ++b;
	return b;
}

__global__ void pairs_kernel(int P, const float2* xy, const float* depth, const uint32_t* incl, const int* radii,
	dim3 grid, uint64_t* keys, uint32_t* vals)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= P || radii[i] <= 0) return;
	uint32_t at = i == 0 ? 0 : incl[i - 1];
	uint2 lo, hi;
	getRect(xy[i], radii[i], lo, hi, grid);
	for (unsigned y = lo.y; y < hi.y; ++y)
		for (unsigned x = lo.x; x < hi.x; ++x) {
			keys[at] = ((uint64_t)(y * grid.x + x) << 32) | __float_as_uint(depth[i]);
			vals[at] = (uint32_t)i;
			++at;
		}
}

__global__ void ranges_kernel(int L, const uint64_t* keys, uint2* ranges)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= L) return;
	const uint32_t t = (uint32_t)(keys[k] >> 32);
	if (k == 0 || (uint32_t)(keys[k - 1] >> 32) != t) ranges[t].x = k;
	if (k == L - 1 || (uint32_t)(keys[k + 1] >> 32) != t) ranges[t].y = k + 1;
}

struct Frame {
	int P = 0, D = 0, M = 0, W = 0, H = 0, sh = -1, aa = 0;
	dim3 grid, block;
	float tan_fovx = 0, tan_fovy = 0, focal_x = 0, focal_y = 0, scale_mod = 1;
	float3 bmin, bmax;
	float *pos = nullptr, *sc = nullptr, *rot = nullptr, *op = nullptr, *col = nullptr, *view = nullptr,
		*proj = nullptr, *cam = nullptr, *depth = nullptr, *cov = nullptr, *rgb = nullptr, *T = nullptr,
		*out = nullptr, *bg = nullptr;
	float2* xy = nullptr;
	float4* con = nullptr;
	int *radii = nullptr, *pick = nullptr;
	uint32_t *touched = nullptr, *incl = nullptr, *vals = nullptr, *vals_s = nullptr, *contrib = nullptr;
	uint64_t *keys = nullptr, *keys_s = nullptr;
	uint2* ranges = nullptr;
	bool* clamped = nullptr;
	void* temp = nullptr;
	size_t temp_bytes = 0;
	long long cap = 0, L = 0;

	// one frame on resident inputs; returns the pair count
	long long run()
	{
		preprocessCUDA<NUM_CHANNELS><<<(P + 255) / 256, 256>>>(P, D, M, pos, pos, nullptr, nullptr, nullptr, nullptr,
			(const glm::vec3*)sc, scale_mod, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f,
			(const glm::vec4*)rot, op, sh < 0 ? nullptr : col, clamped, nullptr, sh < 0 ? col : nullptr, view, proj,
			(const glm::vec3*)cam, W, H, tan_fovx, tan_fovy, focal_x, focal_y, radii, xy, depth, cov, rgb, con, grid,
			touched, false, nullptr, bmin, bmax, aa != 0, 0.0f, false, false, false, nullptr, 0.0f, nullptr);
		size_t need = 0;
		cub::DeviceScan::InclusiveSum(nullptr, need, touched, incl, P);
		grow(need);
		cub::DeviceScan::InclusiveSum(temp, need, touched, incl, P);
		uint32_t total = 0;
		cudaMemcpy(&total, incl + P - 1, 4, cudaMemcpyDeviceToHost);
		L = total;
		const int tiles = grid.x * grid.y;
		cudaMemset(ranges, 0, sizeof(uint2) * tiles);
		if (L > 0) {
			if (L > cap) {
				cudaFree(keys); cudaFree(keys_s); cudaFree(vals); cudaFree(vals_s);
				cap = L + L / 4;
				cudaMalloc(&keys, 8 * cap); cudaMalloc(&keys_s, 8 * cap);
				cudaMalloc(&vals, 4 * cap); cudaMalloc(&vals_s, 4 * cap);
			}
			pairs_kernel<<<(P + 255) / 256, 256>>>(P, xy, depth, incl, radii, grid, keys, vals);
			const int bit = getHigherMsb(tiles);
			cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_s, vals, vals_s, (int)L, 0, 32 + bit);
			grow(need);
			cub::DeviceRadixSort::SortPairs(temp, need, keys, keys_s, vals, vals_s, (int)L, 0, 32 + bit);
			ranges_kernel<<<(int)((L + 255) / 256), 256>>>((int)L, keys_s, ranges);
		}
		if (pick) cudaMemset(pick, 0xff, 4 * (size_t)W * H);
		FORWARD::render(grid, block, ranges, vals_s, W, H, xy, sh < 0 ? col : rgb, con, T, contrib, bg, out, pick);
		return L;
	}

	void grow(size_t need)
	{
		if (need <= temp_bytes) return;
		cudaFree(temp);
		cudaMalloc(&temp, need);
		temp_bytes = need;
	}

	void release()
	{
		void* bufs[] = { pos, sc, rot, op, col, view, proj, cam, depth, cov, rgb, T, out, bg, xy, con, radii, pick,
			touched, incl, vals, vals_s, contrib, keys, keys_s, ranges, clamped, temp };
		for (void* b : bufs)
			if (b) cudaFree(b);
	}
};

}  // namespace refrender

static long long ref_render(int P, const float* pos, const float* scales, const float* rots, const float* opacity,
	const float* colors, int sh_degree, const float* view, const float* proj, const float* campos, int W, int H,
	float tan_fovx, float tan_fovy, float scale_mod, int antialias, const float* box_lo, const float* box_hi,
	const float* bg, int pick, const float* floor_p, float* out, float* final_T_out, int* n_contrib_out, int* pick_out,
	int* radii_out, int reps, float* ms_per_frame)
{
	if (P <= 0 || W <= 0 || H <= 0) return -1;
	refrender::Frame F;
	F.P = P; F.W = W; F.H = H; F.sh = sh_degree; F.aa = antialias;
	F.D = sh_degree < 0 ? 0 : sh_degree;
	F.M = sh_degree < 0 ? 0 : (sh_degree + 1) * (sh_degree + 1);
	F.grid = dim3((W + BLOCK_X - 1) / BLOCK_X, (H + BLOCK_Y - 1) / BLOCK_Y, 1);
	F.block = dim3(BLOCK_X, BLOCK_Y, 1);
	F.tan_fovx = tan_fovx; F.tan_fovy = tan_fovy;
	F.focal_y = H / (2.0f * tan_fovy); F.focal_x = W / (2.0f * tan_fovx);
	F.scale_mod = scale_mod;
	F.bmin = box_lo ? make_float3(box_lo[0], box_lo[1], box_lo[2]) : make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
	F.bmax = box_hi ? make_float3(box_hi[0], box_hi[1], box_hi[2]) : make_float3(FLT_MAX, FLT_MAX, FLT_MAX);
	const size_t ncol = sh_degree < 0 ? 3 * (size_t)P : 3 * (size_t)F.M * P;
	const int tiles = F.grid.x * F.grid.y;
	const size_t np = (size_t)W * H;
	cudaMalloc(&F.pos, 12 * (size_t)P); cudaMalloc(&F.sc, 12 * (size_t)P); cudaMalloc(&F.rot, 16 * (size_t)P);
	cudaMalloc(&F.op, 4 * (size_t)P); cudaMalloc(&F.col, 4 * ncol); cudaMalloc(&F.view, 64); cudaMalloc(&F.proj, 64);
	cudaMalloc(&F.cam, 12); cudaMalloc(&F.depth, 4 * (size_t)P); cudaMalloc(&F.cov, 24 * (size_t)P);
	cudaMalloc(&F.rgb, 12 * (size_t)P); cudaMalloc(&F.xy, 8 * (size_t)P); cudaMalloc(&F.con, 16 * (size_t)P);
	cudaMalloc(&F.radii, 4 * (size_t)P); cudaMalloc(&F.touched, 4 * (size_t)P); cudaMalloc(&F.incl, 4 * (size_t)P);
	cudaMalloc(&F.clamped, 3 * (size_t)P); cudaMalloc(&F.ranges, sizeof(uint2) * tiles);
	cudaMalloc(&F.T, 4 * np); cudaMalloc(&F.contrib, 4 * np); cudaMalloc(&F.out, 12 * np); cudaMalloc(&F.bg, 12);
	if (pick) cudaMalloc(&F.pick, 4 * np);
	cudaMemcpy(F.pos, pos, 12 * (size_t)P, cudaMemcpyHostToDevice);
	cudaMemcpy(F.sc, scales, 12 * (size_t)P, cudaMemcpyHostToDevice);
	cudaMemcpy(F.rot, rots, 16 * (size_t)P, cudaMemcpyHostToDevice);
	cudaMemcpy(F.op, opacity, 4 * (size_t)P, cudaMemcpyHostToDevice);
	cudaMemcpy(F.col, colors, 4 * ncol, cudaMemcpyHostToDevice);
	cudaMemcpy(F.view, view, 64, cudaMemcpyHostToDevice);
	cudaMemcpy(F.proj, proj, 64, cudaMemcpyHostToDevice);
	cudaMemcpy(F.cam, campos, 12, cudaMemcpyHostToDevice);
	const float zero3[3] = { 0.0f, 0.0f, 0.0f };
	cudaMemcpy(F.bg, bg ? bg : zero3, 12, cudaMemcpyHostToDevice);
	// checker floor: the solver's ground statics plus setGroundRender, restored after
	const float keepN[3] = { g_groundN[0], g_groundN[1], g_groundN[2] };
	const float keepH = g_groundHeight;
	if (floor_p) {
		for (int k = 0; k < 3; ++k) g_groundN[k] = floor_p[k];
		g_groundHeight = floor_p[3];
		FORWARD::setGroundRender(true, floor_p + 4, floor_p[7], floor_p[8], view, campos, tan_fovx, tan_fovy);
	}
	long long L = F.run();
	if (reps > 0 && ms_per_frame) {
		cudaEvent_t a, b;
		cudaEventCreate(&a);
		cudaEventCreate(&b);
		cudaDeviceSynchronize();
		cudaEventRecord(a);
		for (int r = 0; r < reps; ++r) L = F.run();
		cudaEventRecord(b);
		cudaEventSynchronize(b);
		float ms = 0.0f;
		cudaEventElapsedTime(&ms, a, b);
		*ms_per_frame = ms / reps;
		cudaEventDestroy(a);
		cudaEventDestroy(b);
	}
	cudaDeviceSynchronize();
	if (floor_p) {
		FORWARD::setGroundRender(false, nullptr, 1.0f, 1.0f, nullptr, nullptr, 1.0f, 1.0f);
		for (int k = 0; k < 3; ++k) g_groundN[k] = keepN[k];
		g_groundHeight = keepH;
	}
	const bool ok = cudaGetLastError() == cudaSuccess;
	if (out) cudaMemcpy(out, F.out, 12 * np, cudaMemcpyDeviceToHost);
	if (final_T_out) cudaMemcpy(final_T_out, F.T, 4 * np, cudaMemcpyDeviceToHost);
	if (n_contrib_out) cudaMemcpy(n_contrib_out, F.contrib, 4 * np, cudaMemcpyDeviceToHost);
	if (pick_out && pick) cudaMemcpy(pick_out, F.pick, 4 * np, cudaMemcpyDeviceToHost);
	if (radii_out) cudaMemcpy(radii_out, F.radii, 4 * (size_t)P, cudaMemcpyDeviceToHost);
	F.release();
	return ok ? L : -1;
}

// One frame (sh_degree -1: colours are RGB, colors_precomp; else SH coefficients
// [n][(d+1)^2][3]; floor_p NULL or {normal[3], height, origin[3], checker, fade}).
// Returns the pair count (num_rendered).
__attribute__((visibility("default"))) long long refshim_render(int P, const float* pos, const float* scales,
	const float* rots, const float* opacity, const float* colors, int sh_degree, const float* view, const float* proj,
	const float* campos, int W, int H, float tan_fovx, float tan_fovy, float scale_mod, int antialias,
	const float* box_lo, const float* box_hi, const float* bg, int pick, const float* floor_p, float* out,
	float* final_T_out, int* n_contrib_out, int* pick_out, int* radii_out)
{
	return ref_render(P, pos, scales, rots, opacity, colors, sh_degree, view, proj, campos, W, H, tan_fovx, tan_fovy,
		scale_mod, antialias, box_lo, box_hi, bg, pick, floor_p, out, final_T_out, n_contrib_out, pick_out, radii_out,
		0, nullptr);
}

// The same frame repeated reps times on resident inputs: milliseconds per frame
// (CUDA events around preprocess + scan + pair keys + sort + ranges + render, the
// pair-count readback included as in Rasterizer::forward).
__attribute__((visibility("default"))) long long refshim_render_timed(int P, const float* pos, const float* scales,
	const float* rots, const float* opacity, const float* colors, int sh_degree, const float* view, const float* proj,
	const float* campos, int W, int H, float tan_fovx, float tan_fovy, int reps, float* ms_per_frame)
{
	return ref_render(P, pos, scales, rots, opacity, colors, sh_degree, view, proj, campos, W, H, tan_fovx, tan_fovy,
		1.0f, 0, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, reps,
		ms_per_frame);
}

}  // extern "C"
