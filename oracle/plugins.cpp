/* ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
 *
 * Neuron-model updates of the reference CPU plugins, restated with the same
 * plugin signature (src/nemo/cpu/plugins/neuron_model.h:25-38) and the same
 * floating-point operation order. Built with -ffp-contract=off.
 *
 * Indexing: arrays shared by all types (currents, fstim, recentFiring, fired)
 * are indexed with the simulation index ng = start + nl, per-type arrays
 * (parameters, state, rng) with the type-local index nl. The reference QIF and
 * HH plugins index their per-type arrays with ng (QIF.cpp:67-68, HH.cpp:70-74),
 * which is only defined when the type starts at simulation index 0; in that
 * case both readings coincide. */

#include "oracle.hpp"

#include <cmath>

namespace oracle {

/* Parameter and state indices: src/nemo/plugins/Izhikevich.h:6-15 */
enum { IZ_A, IZ_B, IZ_C, IZ_D, IZ_SIGMA };
enum { IZ_U, IZ_V };

/* src/nemo/cpu/plugins/Izhikevich.cpp:14-98 */
void
update_Izhikevich(unsigned start, unsigned end, unsigned /*cycle*/,
		float* paramBase, size_t paramStride,
		float* stateBase, size_t /*stateHistoryStride*/, size_t stateVarStride,
		unsigned /*fbits*/, unsigned fstim[], RNG rng[],
		float currentEPSP[], float currentIPSP[], float currentExternal[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	const unsigned SUBSTEPS = 4;
	const float SUBSTEP_MULT = 0.25f;

	const float* a = paramBase + IZ_A * paramStride;
	const float* b = paramBase + IZ_B * paramStride;
	const float* c = paramBase + IZ_C * paramStride;
	const float* d = paramBase + IZ_D * paramStride;
	const float* sigma = paramBase + IZ_SIGMA * paramStride;
	float* u_ = stateBase + IZ_U * stateVarStride;
	float* v_ = stateBase + IZ_V * stateVarStride;

	int nn = int(end - start);
#pragma omp parallel for default(shared)
	for(int nl = 0; nl < nn; nl++) {
		unsigned ng = start + nl;
		float I = currentEPSP[ng] + currentIPSP[ng] + currentExternal[ng];
		currentExternal[ng] = 0.0f;
		if(sigma[nl] != 0.0f) {
			I += sigma[nl] * nrand(&rng[nl]);
		}
		fired[ng] = 0;
		float u = u_[nl];
		float v = v_[nl];
		for(unsigned t = 0; t < SUBSTEPS; ++t) {
			if(!fired[ng]) {
				/* double literals: the bracket is evaluated in double */
				v += SUBSTEP_MULT * ((0.04 * v + 5.0) * v + 140.0 - u + I);
				u += SUBSTEP_MULT * (a[nl] * (b[nl] * v - u));
				fired[ng] = v >= 30.0;
			}
		}
		fired[ng] |= fstim[ng];
		fstim[ng] = 0;
		recentFiring[ng] = (recentFiring[ng] << 1) | (uint64_t) fired[ng];
		if(fired[ng]) {
			v = c[nl];
			u += d[nl];
		}
		u_[nl] = u;
		v_[nl] = v;
	}
}

/* src/nemo/plugins/IF_curr_exp.h:4-17 */
enum { LIF_V_REST, LIF_V_RESET, LIF_C_M, LIF_TAU_M, LIF_TAU_REFRAC,
	LIF_TAU_SYN_E, LIF_TAU_SYN_I, LIF_V_THRESH, LIF_I_OFFSET };
enum { LIF_V, LIF_IE, LIF_II, LIF_LASTFIRED };

/* src/nemo/cpu/plugins/IF_curr_exp.cpp:27-122 */
void
update_IF_curr_exp(unsigned start, unsigned end, unsigned /*cycle*/,
		float* paramBase, size_t paramStride,
		float* stateBase, size_t /*stateHistoryStride*/, size_t stateVarStride,
		unsigned /*fbits*/, unsigned fstim[], RNG /*rng*/[],
		float currentEPSP[], float currentIPSP[], float currentExternal[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	const float* p_v_rest = paramBase + LIF_V_REST * paramStride;
	const float* p_c_m = paramBase + LIF_C_M * paramStride;
	const float* p_tau_m = paramBase + LIF_TAU_M * paramStride;
	const float* p_tau_refrac = paramBase + LIF_TAU_REFRAC * paramStride;
	const float* p_tau_syn_E = paramBase + LIF_TAU_SYN_E * paramStride;
	const float* p_tau_syn_I = paramBase + LIF_TAU_SYN_I * paramStride;
	const float* p_I_offset = paramBase + LIF_I_OFFSET * paramStride;
	const float* p_v_reset = paramBase + LIF_V_RESET * paramStride;
	const float* p_v_thresh = paramBase + LIF_V_THRESH * paramStride;
	float* v_ = stateBase + LIF_V * stateVarStride;
	float* Ie_ = stateBase + LIF_IE * stateVarStride;
	float* Ii_ = stateBase + LIF_II * stateVarStride;
	float* lastfired_ = stateBase + LIF_LASTFIRED * stateVarStride;

	int nn = int(end - start);
#pragma omp parallel for default(shared)
	for(int nl = 0; nl < nn; nl++) {
		unsigned ng = start + nl;
		float Ie = ((1.0f - 1.0f / p_tau_syn_E[nl]) * Ie_[nl]) + currentEPSP[ng];
		float Ii = ((1.0f - 1.0f / p_tau_syn_I[nl]) * Ii_[nl]) + currentIPSP[ng];
		float I = Ie + Ii + currentExternal[ng] + p_I_offset[nl];
		Ie_[nl] = Ie;
		Ii_[nl] = Ii;
		currentExternal[ng] = 0.0f;
		float v = v_[nl];
		bool refractory = lastfired_[nl] <= p_tau_refrac[nl];
		if(!refractory) {
			float c_m = p_c_m[nl];
			float v_rest = p_v_rest[nl];
			float tau_m = p_tau_m[nl];
			v += I / c_m + (v_rest - v) / tau_m;
		}
		/* strict '>' on the CPU backend (IF_curr_exp.cpp:107) */
		fired[ng] = (!refractory && v > p_v_thresh[nl]) || fstim[ng];
		fstim[ng] = 0;
		recentFiring[ng] = (recentFiring[ng] << 1) | (uint64_t) fired[ng];
		if(fired[ng]) {
			lastfired_[nl] = 1;
			v_[nl] = p_v_reset[nl];
		} else {
			lastfired_[nl] += 1;
			v_[nl] = v;
		}
	}
}

/* src/nemo/cpu/plugins/QIF.cpp:16-107 (QIF.h: PARAM_A 0, STATE_V 0) */
void
update_QIF(unsigned start, unsigned end, unsigned /*cycle*/,
		float* paramBase, size_t /*paramStride*/,
		float* stateBase, size_t /*stateHistoryStride*/, size_t /*stateVarStride*/,
		unsigned /*fbits*/, unsigned fstim[], RNG /*rng*/[],
		float currentEPSP[], float currentIPSP[], float currentExternal[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	const float* a0 = paramBase;
	float* v_ = stateBase;

	float dt = 0.1f;
	float a1 = 0.5f * dt;
	float a2 = dt;
	float bb1 = dt / 6.0f;
	unsigned int inc_max = (unsigned int)(1 / dt); /* 10 */

	for(unsigned n = start; n < end; ++n) {
		unsigned nl = n - start;
		float Excit = currentEPSP[n];
		float Inhib = currentIPSP[n];
		float Exter = currentExternal[n];
		currentExternal[n] = 0.0f;
		fired[n] = 0;
		float v = v_[nl];
		float a = a0[nl];
		for(unsigned t = 0; t < inc_max; ++t) {
			if(!fired[n]) {
				float I = Excit + Inhib + Exter;
				I = I * 0.015f;
				float k1 = a * v * (v - 1) + I;
				float x2 = v + a1 * k1;
				float k2 = a * x2 * (x2 - 1) + I;
				float x3 = v + a1 * k2;
				float k3 = a * x3 * (x3 - 1) + I;
				float x4 = v + a2 * k3;
				float k4 = a * x4 * (x4 - 1) + I;
				v = v + bb1 * (k1 + 2 * k2 + 2 * k3 + k4);
				fired[n] = v >= 1;
			}
		}
		fired[n] |= fstim[n];
		fstim[n] = 0;
		recentFiring[n] = (recentFiring[n] << 1) | (uint64_t) fired[n];
		if(fired[n]) {
			v = 0;
		}
		v_[nl] = v;
	}
}

/* src/nemo/cpu/plugins/HH.cpp:14-137. The reference calls exp() on float
 * arguments from C++ <math.h>, which resolves to the float overload and thus
 * to libm expf; the restatement calls expf directly. */
void
update_HH(unsigned start, unsigned end, unsigned cycle,
		float* /*paramBase*/, size_t /*paramStride*/,
		float* stateBase, size_t /*stateHistoryStride*/, size_t stateVarStride,
		unsigned /*fbits*/, unsigned fstim[], RNG /*rng*/[],
		float currentEPSP[], float currentIPSP[], float currentExternal[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	float* v_ = stateBase + 0 * stateVarStride;
	float* n_ = stateBase + 1 * stateVarStride;
	float* m_ = stateBase + 2 * stateVarStride;
	float* h_ = stateBase + 3 * stateVarStride;
	float* dir_ = stateBase + 4 * stateVarStride;

	float dt = 0.001f;
	float gNa = 120.0f;
	float gK = 36.0f;
	float gL = 0.3f;
	float ENa = 115.0f - 65.0f;
	float EK = -12.0f - 65.0f;
	float EL = 10.6f - 65.0f;
	float C = 1.0f;
	float RevE = 0.0f;
	float RevI = -70.0f;
	int inc_max = (int)(1 / dt); /* 999 */

	for(unsigned nn = start; nn < end; ++nn) {
		unsigned nl = nn - start;
		float v = v_[nl];
		float n = n_[nl];
		float m = m_[nl];
		float h = h_[nl];
		float dir = dir_[nl];
		float Excit = currentEPSP[nn];
		float Inhib = currentIPSP[nn];
		float Exter = currentExternal[nn];
		currentExternal[nn] = 0.0f;
		fired[nn] = 0;
		for(unsigned t = 0; t < unsigned(inc_max); ++t) {
			float I = (Excit * (RevE - v)) + (Inhib * ((RevI - v) / -1)) + Exter;
			float alphan = (0.1f - 0.01f * (v + 65.0f)) / (expf(1.0f - 0.1f * (v + 65.0f)) - 1.0f);
			float alpham = (2.5f - 0.1f * (v + 65.0f)) / (expf(2.5f - 0.1f * (v + 65.0f)) - 1.0f);
			float alphah = 0.07f * expf(-(v + 65.0f) / 20.0f);
			float betan = 0.125f * expf(-(v + 65.0f) / 80.0f);
			float betam = 4.0f * expf(-(v + 65.0f) / 18.0f);
			float betah = 1.0f / (expf(3.0f - 0.1f * (v + 65.0f)) + 1.0f);
			m = m + dt * (alpham * (1.0f - m) - betam * m);
			n = n + dt * (alphan * (1.0f - n) - betan * n);
			h = h + dt * (alphah * (1.0f - h) - betah * h);
			float Ik = gNa * (m * m * m) * h * (v - ENa) + gK * (n * n * n * n) * (v - EK) + gL * (v - EL);
			float newv = v + dt * (-Ik + I) / C;
			float new_dir = (newv - v);
			float change = (dir < 0) | (newv < -45) ? 0 : new_dir;
			dir = new_dir;
			if(!fired[nn] && cycle >= 10)
				fired[nn] = change < -0.000000001;
			v = newv;
		}
		fired[nn] |= fstim[nn];
		fstim[nn] = 0;
		recentFiring[nn] = (recentFiring[nn] << 1) | (uint64_t) fired[nn];
		v_[nl] = v;
		n_[nl] = n;
		m_[nl] = m;
		h_[nl] = h;
		dir_[nl] = dir;
	}
}

/* src/nemo/cpu/plugins/PoissonSource.cpp:6-30 (one parameter: rate) */
void
update_PoissonSource(unsigned start, unsigned end, unsigned /*cycle*/,
		float* paramBase, size_t /*paramStride*/,
		float* /*stateBase*/, size_t /*stateHistoryStride*/, size_t /*stateVarStride*/,
		unsigned /*fbits*/, unsigned fstim[], RNG rng[],
		float /*currentEPSP*/[], float /*currentIPSP*/[], float /*currentExternal*/[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	const float* rate = paramBase;
	for(unsigned ng = start, nl = 0U; ng < end; ng++, nl++) {
		unsigned p0 = unsigned(rate[nl] * float(1 << 16));
		unsigned p1 = urand(&rng[nl]) & 0xffff;
		fired[ng] = p1 < p0 || fstim[ng];
		fstim[ng] = 0;
		recentFiring[ng] = (recentFiring[ng] << 1) | (uint64_t) fired[ng];
	}
}

/* src/nemo/cpu/plugins/Input.cpp:6-26 */
void
update_Input(unsigned start, unsigned end, unsigned /*cycle*/,
		float* /*paramBase*/, size_t /*paramStride*/,
		float* /*stateBase*/, size_t /*stateHistoryStride*/, size_t /*stateVarStride*/,
		unsigned /*fbits*/, unsigned fstim[], RNG /*rng*/[],
		float /*currentEPSP*/[], float /*currentIPSP*/[], float /*currentExternal*/[],
		uint64_t recentFiring[], unsigned fired[], void* /*rcm*/)
{
	for(unsigned n = start; n < end; n++) {
		fired[n] = fstim[n];
		fstim[n] = 0;
		recentFiring[n] = (recentFiring[n] << 1) | (uint64_t) fired[n];
	}
}

/* Descriptor fields of src/nemo/plugins/{Izhikevich,IF_curr_exp,QIF,HH,
 * PoissonSource,Input}.ini. A name without a descriptor fails like the
 * reference's .ini lookup (src/nemo/NeuronType.cpp:40-72). */
NeuronType
neuronType(const std::string& name)
{
	struct Row { const char* name; unsigned p, s, mp; bool nrand; cpu_update_neurons_t* fn; };
	static const Row rows[] = {
		{"Izhikevich", 5, 2, 1, true, update_Izhikevich},
		{"IF_curr_exp", 9, 4, 0, false, update_IF_curr_exp},
		{"QIF", 1, 1, 0, false, update_QIF},
		{"HH", 0, 5, 0, false, update_HH},
		{"PoissonSource", 1, 0, 0, true, update_PoissonSource},
		{"Input", 0, 0, 0, false, update_Input},
	};
	for(const Row& r : rows) {
		if(name == r.name) {
			NeuronType t;
			t.name = r.name;
			t.nParam = r.p;
			t.nState = r.s;
			t.membranePotential = r.mp;
			t.history = 1;
			t.nrand = r.nrand;
			t.update = r.fn;
			return t;
		}
	}
	throw Error(NEMO_INVALID_INPUT, "Could not find .ini file for plugin " + name);
}

} // namespace oracle
