/* ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
 *
 * Fixed point, RNG, STDP rule and neuron-model updates of the reference CPU
 * backend, restated. Built with -ffp-contract=off so that every float/double
 * operation is rounded individually, as in the reference build. */

#include "oracle.hpp"

#include <cmath>
#include <cstdlib>
#include <random>
#include <sstream>

namespace oracle {

/* src/nemo/fixedpoint.cpp:17-29. Overflow raises a plain std::runtime_error,
 * which the C ABI reports as NEMO_UNKNOWN_ERROR (nemo_c.cpp:48-49). */
fix_t
fx_toFix(float f, unsigned fbits)
{
	if(std::abs(int(f)) >= 1 << (31 - fbits)) {
		std::ostringstream msg;
		msg << "Fixed-point overflow. Value " << f
			<< " does not fit into fixed-point format Q"
			<< 31 - fbits << "." << fbits;
		throw std::runtime_error(msg.str());
	}
	return static_cast<fix_t>(f * (1 << fbits));
}

/* src/nemo/fixedpoint.cpp:32-36 */
float
fx_toFloat(fix_t v, unsigned fbits)
{
	return float(v) / float(1 << fbits);
}

/* src/nemo/fixedpoint.cpp:40-49 (NEMO_WEIGHT_FIXED_POINT_SATURATION is ON,
 * src/nemo/CMakeLists.txt:1) */
float
wfx_toFloat(wfix_t v, unsigned fbits)
{
	v = std::min(v, wfix_t(fx_max));
	v = std::max(v, wfix_t(fx_min));
	return float(v) / float(1 << fbits);
}

/* src/nemo/RNG.cpp:39-62. The seeds come from a default-seeded mt19937 passed
 * through boost::uniform_int<unsigned long>(0, 0x7fffffff). Boost's published
 * uniform_int algorithm (>= 1.47) maps a 32-bit engine onto [0, 2^31) with a
 * bucket size of 2, i.e. mt() >> 1. std::mt19937 is the same engine with the
 * same default seed (5489). */
void
initialiseRng(unsigned minIdx, unsigned maxIdx, std::vector<RNG>& rngs)
{
	if(!(minIdx <= maxIdx)) {
		throw Error(NEMO_LOGIC_ERROR, "Invalid neuron range when initialising RNG");
	}
	std::mt19937 mt;
	for(unsigned i = 0; i < 4 * minIdx; ++i) {
		mt();
	}
	for(unsigned g = minIdx; g <= maxIdx; ++g) {
		RNG& seeds = rngs.at(g - minIdx);
		for(unsigned plane = 0; plane < 4; ++plane) {
			seeds.state[plane] = unsigned(mt() >> 1);
		}
	}
}

/* ---- StdpFunction: src/nemo/StdpFunction.cpp:9-107 ---- */

StdpFunction::StdpFunction(const std::vector<float>& pre, const std::vector<float>& post,
		float minE, float maxE, float minI, float maxI) :
	prefire(pre), postfire(post), minE(minE), maxE(maxE), minI(minI), maxI(maxI)
{
	if(maxI > 0.0f || minI > 0.0f) {
		throw Error(NEMO_INVALID_INPUT, "STDP function should not have positive limits for inhibitory synapses");
	}
	if(maxE < 0.0f || minE < 0.0f) {
		throw Error(NEMO_INVALID_INPUT, "STDP function should not have negative limits for inhibitory synapses");
	}
	if(maxE < minE) {
		throw Error(NEMO_INVALID_INPUT, "STDP should have maximum excitatory weight >= minimum excitatory weight");
	}
	if(maxI > minI) {
		throw Error(NEMO_INVALID_INPUT, "STDP should have abs(maximum inhibitory weight) >= abs(minimum inhibitory weight)");
	}
	if(prefire.size() + postfire.size() > 64) {
		throw Error(NEMO_INVALID_INPUT, "size of STDP window too large");
	}
}

void
StdpFunction::verifyDynamicWindowLength(unsigned d_max) const
{
	if(d_max + postfire.size() > 64) {
		throw Error(NEMO_INVALID_INPUT, "Max delay + postfire part of STDP function must be <= 64");
	}
}

/* LSB = end of the window: the postfire part reversed, then the prefire part
 * (StdpFunction.cpp:51-68) */
uint64_t
StdpFunction::getBits(bool (*pred)(float)) const
{
	uint64_t bits = 0;
	int n = 0;
	for(auto f = postfire.rbegin(); f != postfire.rend(); ++f, ++n) {
		if(pred(*f)) {
			bits |= uint64_t(1) << n;
		}
	}
	for(auto f = prefire.begin(); f != prefire.end(); ++f, ++n) {
		if(pred(*f)) {
			bits |= uint64_t(1) << n;
		}
	}
	return bits;
}

static bool potentiation(float x) { return x > 0.0f; }
static bool depression(float x) { return x < 0.0f; }
uint64_t StdpFunction::potentiationBits() const { return getBits(potentiation); }
uint64_t StdpFunction::depressionBits() const { return getBits(depression); }

/* 64-bit shifts whose count can reach 64. The reference evaluates them with
 * the x86-64 shift instruction, which uses the count modulo 64; that is the
 * behaviour restated here (and by the B200 kernels). */
static inline uint64_t shl64(uint64_t x, unsigned n) { return x << (n & 63); }
static inline uint64_t shr64(uint64_t x, unsigned n) { return x >> (n & 63); }

/* ---- StdpProcess: src/nemo/StdpProcess.cpp:20-46 ---- */
StdpProcess::StdpProcess(const StdpFunction& fn, unsigned fbits) :
	m_minE(fx_toFix(fn.minE, fbits)),
	m_maxE(fx_toFix(fn.maxE, fbits)),
	m_minI(fx_toFix(fn.minI, fbits)),
	m_maxI(fx_toFix(fn.maxI, fbits))
{
	for(float f : fn.prefire) m_fnPre.push_back(fx_toFix(f, fbits));
	for(float f : fn.postfire) m_fnPost.push_back(fx_toFix(f, fbits));
	m_potentiationBits = fn.potentiationBits();
	m_depressionBits = fn.depressionBits();
	unsigned prePostWindow = unsigned(fn.prefire.size());
	m_postPreWindow = int(fn.postfire.size());
	m_prePostBits = shl64(~shl64(~uint64_t(0), prePostWindow), m_postPreWindow);
	m_postPreBits = ~shl64(~uint64_t(0), m_postPreWindow);
	m_postFireMask = shl64(uint64_t(1), m_postPreWindow);
}

/* StdpProcess.cpp:68-74 */
unsigned
StdpProcess::closestPreFire(uint64_t arrivals) const
{
	uint64_t valid = arrivals & m_prePostBits;
	if(!valid) return NONE;
	return unsigned(__builtin_ctzll(shr64(valid, m_postPreWindow)));
}

/* StdpProcess.cpp:77-83 */
unsigned
StdpProcess::closestPostFire(uint64_t arrivals) const
{
	uint64_t valid = arrivals & m_postPreBits;
	if(!valid) return NONE;
	return unsigned(__builtin_clzll(shl64(valid, 64 - m_postPreWindow)));
}

/* StdpProcess.cpp:87-113 */
fix_t
StdpProcess::updateRegion(uint64_t arrivals) const
{
	fix_t w_diff = 0;
	if(arrivals) {
		unsigned dt_pre = closestPreFire(arrivals);
		unsigned dt_post = closestPostFire(arrivals);
		if(dt_pre < dt_post) {
			w_diff = m_fnPre.at(dt_pre);
		} else if(dt_post < dt_pre) {
			w_diff = m_fnPost.at(dt_post);
		}
	}
	return w_diff;
}

/* StdpProcess.cpp:116-124 */
fix_t
StdpProcess::weightChange(uint64_t preFiring) const
{
	uint64_t p_spikes = preFiring & m_potentiationBits;
	uint64_t d_spikes = preFiring & m_depressionBits;
	return updateRegion(p_spikes) + updateRegion(d_spikes);
}

/* StdpProcess.cpp:128-138: clamp, and synapses stick at zero */
fix_t
StdpProcess::updatedWeight(fix_t w_old, fix_t w_diff) const
{
	fix_t w_new = 0;
	if(w_old > 0) {
		w_new = std::min(m_maxE, std::max(fix_t(uint32_t(w_old) + uint32_t(w_diff)), m_minE));
	} else if(w_old < 0) {
		w_new = std::min(m_minI, std::max(fix_t(uint32_t(w_old) + uint32_t(w_diff)), m_maxI));
	}
	return w_new;
}

/* ---- Configuration defaults: src/nemo/ConfigurationImpl.cpp:19-30 ---- */
Configuration::Configuration() :
	logging(false), writeOnlySynapses(false), fractionalBits(20),
	backend(NEMO_BACKEND_CPU), cudaDevice(-1),
	description("CPU backend (oracle restatement)"), hasStdp(false)
{
}

} // namespace oracle

/* ---- RNG: src/nemo/RNG.cpp:10-34 ---- */

extern "C" unsigned
urand(oracle::RNG* rng)
{
	unsigned t = (rng->state[0] ^ (rng->state[0] << 11));
	rng->state[0] = rng->state[1];
	rng->state[1] = rng->state[2];
	rng->state[2] = rng->state[3];
	rng->state[3] = (rng->state[3] ^ (rng->state[3] >> 19)) ^ (t ^ (t >> 8));
	return rng->state[3];
}

/* Box-Muller, only the sine branch; libm sinf/logf/sqrtf of the host glibc */
extern "C" float
nrand(oracle::RNG* rng)
{
	float a = urand(rng) * 1.4629180792671596810513378043098e-9f;
	float b = urand(rng) * 0.00000000023283064365386962890625f;
	float r = sqrtf(-2 * logf(1 - b));
	return sinf(a) * r;
}
