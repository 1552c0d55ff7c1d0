/* ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * One C surface over the fixed-point conversions and the STDP process,
 * compiled twice: into the oracle library against the restatement
 * (oracle/core.cpp), and with PIN_REFERENCE into oracle/_ref/libnemo_stdp_ref.so
 * against the reference's own sources src/nemo/{fixedpoint,StdpFunction,
 * StdpProcess}.cpp (oracle/Makefile), so that tests/test_oracle_pins.py can
 * run both on the same inputs. Status 0 = ok, 1 = the call threw. */

#include <cstdint>
#include <exception>
#include <vector>

#ifdef PIN_REFERENCE
#include "StdpFunction.hpp"
#include "StdpProcess.hpp"
#include "fixedpoint.hpp"
namespace pin {
typedef nemo::StdpFunction Function;
typedef nemo::StdpProcess Process;
inline fix_t toFix(float f, unsigned b) { return ::fx_toFix(f, b); }
inline float toFloat(fix_t v, unsigned b) { return ::fx_toFloat(v, b); }
inline float wideToFloat(wfix_t v, unsigned b) { return ::wfx_toFloat(v, b); }
inline fix_t mul(fix_t a, fix_t c, unsigned b) { return ::fx_mul(a, c, b); }
inline fix_t change(const Process& p, uint64_t s) { return p.weightChange(s, 0, 0); }
}
#else
#include "oracle.hpp"
namespace pin {
typedef oracle::StdpFunction Function;
typedef oracle::StdpProcess Process;
typedef oracle::fix_t fix_t;
typedef oracle::wfix_t wfix_t;
inline fix_t toFix(float f, unsigned b) { return oracle::fx_toFix(f, b); }
inline float toFloat(fix_t v, unsigned b) { return oracle::fx_toFloat(v, b); }
inline float wideToFloat(wfix_t v, unsigned b) { return oracle::wfx_toFloat(v, b); }
inline fix_t mul(fix_t a, fix_t c, unsigned b) { return oracle::fx_mul(a, c, b); }
inline fix_t change(const Process& p, uint64_t s) { return p.weightChange(s); }
}
#endif

extern "C" {

int
pin_fx_to_fix(const float* f, size_t n, unsigned fbits, int32_t* out, uint8_t* threw)
{
	for(size_t k = 0; k < n; ++k) {
		try {
			out[k] = pin::toFix(f[k], fbits);
			threw[k] = 0;
		} catch(const std::exception&) {
			out[k] = 0;
			threw[k] = 1;
		}
	}
	return 0;
}

void
pin_fx_to_float(const int32_t* v, size_t n, unsigned fbits, float* out)
{
	for(size_t k = 0; k < n; ++k) out[k] = pin::toFloat(v[k], fbits);
}

void
pin_wfx_to_float(const int64_t* v, size_t n, unsigned fbits, float* out)
{
	for(size_t k = 0; k < n; ++k) out[k] = pin::wideToFloat(v[k], fbits);
}

void
pin_fx_mul(const int32_t* a, const int32_t* b, size_t n, unsigned fbits, int32_t* out)
{
	for(size_t k = 0; k < n; ++k) out[k] = pin::mul(a[k], b[k], fbits);
}

/* An STDP process from the function's two windows and four limits, or null
 * when the function is rejected */
void*
pin_stdp_new(const float* pre, size_t npre, const float* post, size_t npost, float minE, float maxE, float minI,
		float maxI, unsigned fbits)
{
	try {
		pin::Function fn(std::vector<float>(pre, pre + npre), std::vector<float>(post, post + npost), minE, maxE,
				minI, maxI);
		return new pin::Process(fn, fbits);
	} catch(const std::exception&) {
		return nullptr;
	}
}

void pin_stdp_delete(void* p) { delete static_cast<pin::Process*>(p); }

/* the function's potentiation and depression bit masks */
int
pin_stdp_bits(const float* pre, size_t npre, const float* post, size_t npost, uint64_t out[2])
{
	try {
		pin::Function fn(std::vector<float>(pre, pre + npre), std::vector<float>(post, post + npost), 0.0f, 1.0f,
				0.0f, -1.0f);
		out[0] = fn.potentiationBits();
		out[1] = fn.depressionBits();
		return 0;
	} catch(const std::exception&) {
		return 1;
	}
}

void
pin_stdp_weight_change(const void* p, const uint64_t* spikes, size_t n, int32_t* out)
{
	const pin::Process& proc = *static_cast<const pin::Process*>(p);
	for(size_t k = 0; k < n; ++k) out[k] = pin::change(proc, spikes[k]);
}

void
pin_stdp_updated_weight(const void* p, const int32_t* wOld, const int32_t* wDiff, size_t n, int32_t* out)
{
	const pin::Process& proc = *static_cast<const pin::Process*>(p);
	for(size_t k = 0; k < n; ++k) out[k] = proc.updatedWeight(wOld[k], wDiff[k]);
}

} // extern "C"
