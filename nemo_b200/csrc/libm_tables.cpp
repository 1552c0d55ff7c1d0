/* Correction tables that let the device reproduce the host glibc sinf/logf
 * results of the reference's thalamic-noise generator bit for bit (see
 * libm_match.cuh for the method). Built once per process on the host with all
 * available cores and cached on disk, keyed by the glibc version.
 *
 * This is calibration data, not a CPU path: the tables record, for each of
 * the 83886081 inputs the RNG can produce, how glibc's rounding differs from
 * the device candidate. The noise itself is computed by the kernels. */

#include "libm_tables.hpp"

#include <gnu/libc-version.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.hpp"
#include "libm_match.cuh"

namespace nemo_b200 {

using namespace libm;

static const uint32_t FILE_MAGIC = 0x4e4d4c54u; /* "NMLT" */
static const uint32_t FILE_VERSION = 1u;

static uint32_t
codeFor(float glibc, float cand)
{
	uint32_t g = f2u(glibc), c = f2u(cand);
	if(g == c) return 0u;
	if(g == c + 1u) return 1u;
	if(g == c - 1u) return 2u;
	return 3u;
}

static void
buildRange(uint32_t w0, uint32_t w1, uint32_t* sinT, uint32_t* logT, unsigned long* bad)
{
	unsigned long nbad = 0;
	for(uint32_t w = w0; w < w1; ++w) {
		uint32_t ws = 0, wl = 0;
		for(uint32_t k = 0; k < 16; ++k) {
			uint32_t idx = w * 16 + k;
			if(idx >= TABLE_ENTRIES) break;
			float fu = libm_value(idx);
			float a = sin_argument(fu);
			float y = log_argument(fu);
			volatile float gs = sinf(a);
			volatile float gl = logf(y);
			uint32_t cs = codeFor(gs, sin_candidate(a));
			uint32_t cl = codeFor(gl, log_candidate(y));
			if(cs == 3u || cl == 3u) nbad++;
			ws |= (cs & 3u) << (2 * k);
			wl |= (cl & 3u) << (2 * k);
		}
		sinT[w] = ws;
		logT[w] = wl;
	}
	*bad = nbad;
}

static std::string
cachePath()
{
	std::string dir;
	if(const char* env = getenv("NEMO_B200_CACHE_DIR")) {
		dir = env;
	} else {
		Dl_info info;
		if(dladdr((void*) &cachePath, &info) && info.dli_fname) {
			std::string lib = info.dli_fname;
			size_t slash = lib.rfind('/');
			dir = (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/data";
		} else {
			dir = "data";
		}
	}
	return dir + "/libm_tables_v1_glibc-" + gnu_get_libc_version() + ".bin";
}

static bool
loadCache(const std::string& path, LibmTables& t)
{
	FILE* f = fopen(path.c_str(), "rb");
	if(!f) return false;
	uint32_t hdr[3] = {0, 0, 0};
	char ver[32] = {0};
	bool ok = fread(hdr, sizeof(hdr), 1, f) == 1 && fread(ver, sizeof(ver), 1, f) == 1
		&& hdr[0] == FILE_MAGIC && hdr[1] == FILE_VERSION && hdr[2] == TABLE_WORDS
		&& strncmp(ver, gnu_get_libc_version(), sizeof(ver)) == 0;
	if(ok) {
		t.sinCodes.resize(TABLE_WORDS);
		t.logCodes.resize(TABLE_WORDS);
		ok = fread(t.sinCodes.data(), 4, TABLE_WORDS, f) == TABLE_WORDS
			&& fread(t.logCodes.data(), 4, TABLE_WORDS, f) == TABLE_WORDS;
	}
	fclose(f);
	return ok;
}

static void
saveCache(const std::string& path, const LibmTables& t)
{
	size_t slash = path.rfind('/');
	if(slash != std::string::npos) {
		mkdir(path.substr(0, slash).c_str(), 0755);
	}
	std::string tmp = path + ".tmp." + std::to_string(getpid());
	FILE* f = fopen(tmp.c_str(), "wb");
	if(!f) return; /* read-only location: keep the in-memory tables */
	uint32_t hdr[3] = {FILE_MAGIC, FILE_VERSION, TABLE_WORDS};
	char ver[32] = {0};
	strncpy(ver, gnu_get_libc_version(), sizeof(ver) - 1);
	bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 && fwrite(ver, sizeof(ver), 1, f) == 1
		&& fwrite(t.sinCodes.data(), 4, TABLE_WORDS, f) == TABLE_WORDS
		&& fwrite(t.logCodes.data(), 4, TABLE_WORDS, f) == TABLE_WORDS;
	ok = (fclose(f) == 0) && ok;
	if(ok) {
		rename(tmp.c_str(), path.c_str());
	} else {
		remove(tmp.c_str());
	}
}

LibmTables
buildLibmTables()
{
	LibmTables t;
	t.sinCodes.assign(TABLE_WORDS, 0);
	t.logCodes.assign(TABLE_WORDS, 0);
	unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
	std::vector<std::thread> pool;
	std::vector<unsigned long> bad(nthreads, 0);
	uint32_t per = (TABLE_WORDS + nthreads - 1) / nthreads;
	for(unsigned i = 0; i < nthreads; ++i) {
		uint32_t w0 = std::min<uint32_t>(TABLE_WORDS, i * per);
		uint32_t w1 = std::min<uint32_t>(TABLE_WORDS, w0 + per);
		pool.emplace_back(buildRange, w0, w1, t.sinCodes.data(), t.logCodes.data(), &bad[i]);
	}
	for(auto& th : pool) th.join();
	unsigned long nbad = 0;
	for(unsigned long b : bad) nbad += b;
	if(nbad) {
		fail(NEMO_LOGIC_ERROR, "libm correction tables: " + std::to_string(nbad)
				+ " inputs differ from glibc by more than one unit in the last place");
	}
	return t;
}

const LibmTables&
libmTables()
{
	static std::mutex lock;
	static LibmTables tables;
	static bool ready = false;
	std::lock_guard<std::mutex> guard(lock);
	if(!ready) {
		std::string path = cachePath();
		if(!loadCache(path, tables)) {
			tables = buildLibmTables();
			saveCache(path, tables);
		}
		ready = true;
	}
	return tables;
}

std::string
libmCachePath()
{
	return cachePath();
}

/* ---- expf exceptions (the HH plugin's exp, src/nemo/cpu/plugins/HH.cpp:92-98) ---- */

static const uint32_t EXP_MAGIC = 0x4e4d4558u; /* "NMEX" */
static const uint32_t EXP_VERSION = 2u;

static std::string
expCachePath()
{
	std::string p = cachePath();
	size_t slash = p.rfind('/');
	std::string dir = slash == std::string::npos ? std::string(".") : p.substr(0, slash);
	return dir + "/expf_exceptions_v2_glibc-" + gnu_get_libc_version() + ".bin";
}

struct ExpPart {
	std::vector<uint32_t> keys, values;
	uint32_t nearUnits = 0;
	unsigned long bad = 0;
};

static void
buildExpRange(uint32_t lo, uint32_t hi, unsigned stride, unsigned offset, ExpPart* out)
{
	for(uint64_t u = uint64_t(lo) + offset; u <= hi; u += stride) {
		const float x = u2f(uint32_t(u));
		volatile float g = expf(x);
		const double c = exp_candidate_d(x);
		const float r = float(c);
		if(f2u(g) != f2u(r)) {
			const int64_t d = int64_t(f2u(g)) - int64_t(f2u(r));
			if(d != 1 && d != -1) out->bad++;
			out->keys.push_back(uint32_t(u));
			out->values.push_back(f2u(g));
			out->nearUnits = std::max(out->nearUnits, exp_midpoint_units(c));
		}
	}
}

static ExpExceptions
buildExpExceptions()
{
	unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
	std::vector<ExpPart> parts(2 * nthreads);
	std::vector<std::thread> pool;
	const uint32_t posHi = f2u(89.0f), negLo = 0x80000000u, negHi = f2u(-104.0f);
	for(unsigned i = 0; i < nthreads; ++i) {
		pool.emplace_back(buildExpRange, 0u, posHi, nthreads, i, &parts[i]);
		pool.emplace_back(buildExpRange, negLo, negHi, nthreads, i, &parts[nthreads + i]);
	}
	for(auto& th : pool) th.join();
	ExpExceptions e;
	std::vector<std::pair<uint32_t, uint32_t>> all;
	unsigned long bad = 0;
	for(const ExpPart& p : parts) {
		for(size_t k = 0; k < p.keys.size(); ++k) all.emplace_back(p.keys[k], p.values[k]);
		e.nearUnits = std::max(e.nearUnits, p.nearUnits);
		bad += p.bad;
	}
	e.tau = double(e.nearUnits) / double(1u << 29);
	if(bad) {
		fail(NEMO_LOGIC_ERROR, "expf exceptions: " + std::to_string(bad)
				+ " inputs differ from glibc by more than one unit in the last place");
	}
	std::sort(all.begin(), all.end());
	for(const auto& kv : all) {
		e.keys.push_back(kv.first);
		e.values.push_back(kv.second);
	}
	return e;
}

static bool
loadExpCache(const std::string& path, ExpExceptions& e)
{
	FILE* f = fopen(path.c_str(), "rb");
	if(!f) return false;
	uint32_t hdr[3] = {0, 0, 0};
	char ver[32] = {0};
	double tau = 0;
	bool ok = fread(hdr, sizeof(hdr), 1, f) == 1 && fread(ver, sizeof(ver), 1, f) == 1
		&& fread(&tau, sizeof(tau), 1, f) == 1
		&& hdr[0] == EXP_MAGIC && hdr[1] == EXP_VERSION
		&& strncmp(ver, gnu_get_libc_version(), sizeof(ver)) == 0;
	if(ok) {
		e.keys.resize(hdr[2]);
		e.values.resize(hdr[2]);
		e.tau = tau;
		e.nearUnits = uint32_t(tau * double(1u << 29) + 0.5);
		ok = fread(e.keys.data(), 4, hdr[2], f) == hdr[2] && fread(e.values.data(), 4, hdr[2], f) == hdr[2];
	}
	fclose(f);
	return ok;
}

static void
saveExpCache(const std::string& path, const ExpExceptions& e)
{
	size_t slash = path.rfind('/');
	if(slash != std::string::npos) {
		mkdir(path.substr(0, slash).c_str(), 0755);
	}
	std::string tmp = path + ".tmp." + std::to_string(getpid());
	FILE* f = fopen(tmp.c_str(), "wb");
	if(!f) return;
	const uint32_t n = uint32_t(e.keys.size());
	uint32_t hdr[3] = {EXP_MAGIC, EXP_VERSION, n};
	char ver[32] = {0};
	strncpy(ver, gnu_get_libc_version(), sizeof(ver) - 1);
	bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 && fwrite(ver, sizeof(ver), 1, f) == 1
		&& fwrite(&e.tau, sizeof(e.tau), 1, f) == 1
		&& fwrite(e.keys.data(), 4, n, f) == n && fwrite(e.values.data(), 4, n, f) == n;
	ok = (fclose(f) == 0) && ok;
	if(ok) {
		rename(tmp.c_str(), path.c_str());
	} else {
		remove(tmp.c_str());
	}
}

/* Insert every (key, value) pair by linear probing into a power-of-two table
 * at most one third full; the probe bound is the longest cyclic run of
 * occupied slots plus one. */
static void
buildExpSlots(ExpExceptions& e)
{
	uint32_t bits = 4;
	while((uint64_t(1) << bits) < 3 * uint64_t(e.keys.size())) ++bits;
	const uint32_t size = 1u << bits, mask = size - 1u;
	e.slots.assign(size, uint64_t(LIBM_EXP_EMPTY_KEY));
	for(size_t k = 0; k < e.keys.size(); ++k) {
		uint32_t h = libm::exp_hash(e.keys[k], bits);
		while(uint32_t(e.slots[h]) != LIBM_EXP_EMPTY_KEY) h = (h + 1u) & mask;
		e.slots[h] = uint64_t(e.values[k]) << 32 | e.keys[k];
	}
	/* longest run of occupied slots, wrapping around the end */
	uint32_t first = 0;
	while(first < size && uint32_t(e.slots[first]) != LIBM_EXP_EMPTY_KEY) ++first;
	uint32_t run = 0, longest = 0;
	for(uint32_t k = 1; k <= size; ++k) {
		if(uint32_t(e.slots[(first + k) & mask]) != LIBM_EXP_EMPTY_KEY) {
			longest = std::max(longest, ++run);
		} else {
			run = 0;
		}
	}
	e.slotBits = bits;
	e.slotProbe = longest + 1;
	/* every pair is found by the device's own lookup, with the same bound */
	for(size_t k = 0; k < e.keys.size(); ++k) {
		const float x = u2f(e.keys[k]);
		const float miss = u2f(e.values[k] ^ 1u);
		if(f2u(libm::exp_lookup(x, miss, e.slots.data(), bits, e.slotProbe)) != e.values[k]) {
			fail(NEMO_LOGIC_ERROR, "expf exception hash: key " + std::to_string(e.keys[k]) + " not found");
		}
	}
}

const ExpExceptions&
expExceptions()
{
	static std::mutex lock;
	static ExpExceptions table;
	static bool ready = false;
	std::lock_guard<std::mutex> guard(lock);
	if(!ready) {
		std::string path = expCachePath();
		if(!loadExpCache(path, table)) {
			table = buildExpExceptions();
			saveExpCache(path, table);
		}
		buildExpSlots(table);
		ready = true;
	}
	return table;
}

} // namespace nemo_b200
