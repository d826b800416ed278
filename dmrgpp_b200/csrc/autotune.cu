// Autotuner of the FP64 H*x launch.
//
// The reference hard-codes its GPU tiling ("tuned" constants for one GH200
// input, BatchedGemmKokkos.h:110-130).  Here each sector is timed under every
// configuration (the persistent two-pass form's tiles and work splits, the
// fused form's where its patches are narrow enough), the fastest is kept,
// and the choice is cached in a text file keyed by a coarse summary of the
// sector's size histogram (work quartiles of the patch dimensions, total
// work, Kronecker terms) and the GPU name, so that sectors of similar shape
// in later sweep steps or runs skip the timing.
#include "dmrgpp_kron.h"
#include "trace.h"
#include "handle.h"
#include "kron_fused.cuh"
#include "kron_persistent.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

using dmrgpp::KronPlan;

// The GPU's name, queried once per device (cudaGetDeviceProperties fills
// every property, which costs far more than a cache lookup of a sweep step).
std::string device_name(int device)
{
	static std::mutex                 mu;
	static std::map<int, std::string> names;
	std::lock_guard<std::mutex>       g(mu);
	auto                              it = names.find(device);
	if (it != names.end())
		return it->second;
	cudaDeviceProp prop {};
	std::string    name = cudaGetDeviceProperties(&prop, device) == cudaSuccess ? prop.name : "unknown";
	names[device]       = name;
	return name;
}

// One line per entry: signature, configuration, items per CTA, the FP64
// apply's microseconds and (optional fifth field) the TF32x3 apply's, -1
// when no TF32x3 form was timed.
bool cache_lookup(const char* path, const std::string& sig, int* cfg, int* ipc, double* us,
                  double* us_tf32x3)
{
	if (!path)
		return false;
	std::ifstream f(path);
	std::string   line;
	bool          found = false;
	while (std::getline(f, line)) {
		std::istringstream in(line);
		std::string        s;
		int                c = -1, i = 0;
		double             t = 0, t32 = -1.0;
		if (in >> s >> c >> i >> t && s == sig && c >= 0 && c < dmrgpp::kNumTileCfgs + dmrgpp::kNumFusedCfgs
		    && i > 0) {
			if (!(in >> t32))
				t32 = -1.0;
			*cfg       = c;
			*ipc       = i;
			*us        = t;
			*us_tf32x3 = t32;
			found      = true; // the last entry wins
		}
	}
	return found;
}

void cache_store(const char* path, const std::string& sig, int cfg, int ipc, double us, double us_tf32x3)
{
	if (!path)
		return;
	std::ofstream f(path, std::ios::app);
	f << sig << ' ' << cfg << ' ' << ipc << ' ' << us << ' ' << us_tf32x3 << '\n';
}

} // namespace

extern "C" {

int dmrgpp_kron_get_config(dmrgpp_kron_handle h, int* cfg, int* items_per_cta)
{
	if (!h || !cfg || !items_per_cta)
		return DMRGPP_INVALID_ARG;
	*cfg           = h->cfg;
	*items_per_cta = h->items_per_cta;
	return DMRGPP_OK;
}

int dmrgpp_kron_set_config(dmrgpp_kron_handle h, int cfg, int items_per_cta)
{
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (cfg < 0 || cfg >= dmrgpp::kNumTileCfgs + dmrgpp::kNumFusedCfgs || items_per_cta < 1
	    || items_per_cta > 64)
		return dmrgpp::handle_fail(h, DMRGPP_INVALID_ARG, "unknown tile configuration");
	int prev = -1;
	cudaGetDevice(&prev);
	if (prev != h->device)
		cudaSetDevice(h->device);
	cudaStreamSynchronize(h->stream);
	const int rc = dmrgpp::configure_schedule(h, cfg, items_per_cta);
	if (prev != h->device && prev >= 0)
		cudaSetDevice(prev);
	return rc;
}

int dmrgpp_kron_autotune(dmrgpp_kron_handle h, const char* cache_path, int reps, int* cfg_out,
                         double* us_out)
{
	DMRGPP_TRACE("dmrgpp_kron_autotune");
	using namespace dmrgpp;
	if (!h)
		return DMRGPP_INVALID_ARG;
	if (reps < 1)
		reps = 10;
	int prev = -1;
	cudaGetDevice(&prev);
	if (prev != h->device)
		cudaSetDevice(h->device);
	struct Restore {
		int dev, prev;
		~Restore()
		{
			if (dev != prev && prev >= 0)
				cudaSetDevice(prev);
		}
	} restore { h->device, prev };

	const std::string sig = dmrgpp::tuning_key(h->plan, device_name(h->device).c_str());
	int               cfg = 0, ipc = 2;
	double            us  = 0.0;
	cudaEvent_t       e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	// minimum over reps of one apply in the handle's current form (or -1)
	auto time_apply = [&]() {
		bool ok = true;
		for (int w = 0; w < 2 && ok; ++w)
			ok = kron_apply_device(h, h->d_x, h->d_y) == DMRGPP_OK;
		double tmin = 1e30;
		for (int r = 0; r < reps && ok; ++r) {
			cudaEventRecord(e0, h->stream);
			ok = kron_apply_device(h, h->d_x, h->d_y) == DMRGPP_OK;
			cudaEventRecord(e1, h->stream);
			cudaEventSynchronize(e1);
			float ms = 0.f;
			cudaEventElapsedTime(&ms, e0, e1);
			tmin = std::min(tmin, double(ms) * 1e3);
		}
		ok = ok && cudaStreamSynchronize(h->stream) == cudaSuccess && h->err_host
		    && *reinterpret_cast<volatile int*>(h->err_host) == 0;
		return ok ? tmin : -1.0;
	};
	// the TF32x3 form (when the handle has one) against the chosen FP64 one,
	// so that a mixed-precision solve can use the faster arithmetic per sector
	auto time_mixed = [&](double fp64_us) {
		h->tuned_fp64_us   = fp64_us;
		h->tuned_tf32x3_us = -1.0;
		if (!h->mixed_ready)
			return;
		const int prec = h->precision;
		h->precision   = DMRGPP_TF32X3;
		h->tuned_tf32x3_us = time_apply();
		h->precision   = prec;
	};
	struct Events {
		cudaEvent_t a, b;
		~Events()
		{
			cudaEventDestroy(a);
			cudaEventDestroy(b);
		}
	} events { e0, e1 };
	const int prec_in = h->precision;
	h->precision      = DMRGPP_FP64; // the configurations are the FP64 forms'
	struct RestorePrecision {
		dmrgpp_kron_handle h;
		int                p;
		~RestorePrecision() { h->precision = p; }
	} restore_prec { h, prec_in };
	double us32 = -1.0;
	if (cache_lookup(cache_path, sig, &cfg, &ipc, &us, &us32)) {
		if (int rc = configure_schedule(h, cfg, ipc))
			return rc;
		h->tuned_fp64_us   = us;
		h->tuned_tf32x3_us = h->mixed_ready ? us32 : -1.0;
		if (h->mixed_ready && us32 < 0) { // an entry made by an FP64 handle
			time_mixed(us);
			cache_store(cache_path, sig, cfg, ipc, us, h->tuned_tf32x3_us);
		}
		if (cfg_out)
			*cfg_out = cfg;
		if (us_out)
			*us_out = us;
		return DMRGPP_OK;
	}

	cudaStreamSynchronize(h->stream);
	const int ipcs[] = { 1, 2, 4 };
	double    best   = -1.0;
	int       bcfg = h->cfg, bipc = h->items_per_cta;
	// fused configurations where the output patches fit in at most two column
	// tiles (wider ones repeat the first product per column tile)
	long long max_l = 0;
	for (size_t p = 0; p < h->plan.np; ++p)
		max_l = std::max(max_l, h->plan.l[p]);
	std::vector<int> cands;
	for (int c = 0; c < kNumTileCfgs; ++c)
		cands.push_back(c);
	for (int f = 0; f < kNumFusedCfgs; ++f)
		if (max_l <= 2LL * fused_shape(f).bn)
			cands.push_back(kNumTileCfgs + f);
	for (int c : cands)
		for (int i : ipcs) {
			if (configure_schedule(h, c, i) != DMRGPP_OK)
				continue;
			const double tmin = time_apply();
			if (tmin >= 0 && (best < 0 || tmin < best)) {
				best = tmin;
				bcfg = c;
				bipc = i;
			}
		}
	if (best < 0)
		return handle_fail(h, DMRGPP_CUDA_ERROR, "autotune: no configuration ran");
	if (int rc = configure_schedule(h, bcfg, bipc))
		return rc;
	time_mixed(best);
	cache_store(cache_path, sig, bcfg, bipc, best, h->tuned_tf32x3_us);
	if (cfg_out)
		*cfg_out = bcfg;
	if (us_out)
		*us_out = best;
	return DMRGPP_OK;
}

int dmrgpp_kron_tuned_times(dmrgpp_kron_handle h, double* fp64_us, double* tf32x3_us)
{
	if (!h || !fp64_us || !tf32x3_us)
		return DMRGPP_INVALID_ARG;
	*fp64_us   = h->tuned_fp64_us;
	*tf32x3_us = h->tuned_tf32x3_us;
	return DMRGPP_OK;
}

} // extern "C"
