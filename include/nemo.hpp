#ifndef NEMO_B200_NEMO_HPP
#define NEMO_B200_NEMO_HPP

/* The reference's C++ API (src/nemo.hpp, src/nemo/Network.hpp,
 * Configuration.hpp, Simulation.hpp, ReadableNetwork.hpp, exception.hpp):
 * the classes nemo::Network, nemo::Configuration and nemo::Simulation with the
 * same method signatures, and nemo::simulation(), implemented header-only over
 * the C ABI of libnemo_b200 (include/nemo.h, include/nemo_b200.h). A failed
 * call throws nemo::exception with the library's status code and message, as
 * the reference's classes do.
 *
 * Differences from the reference: setCpuBackend() throws (the library has no
 * CPU path); the CUDA partition size and the MPI STDP period / reward are
 * kept for the caller to read back but do not change the B200 backend. */

#include <stdint.h>

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <nemo.h>
#include <nemo_b200.h>

namespace nemo {

/* src/nemo/exception.hpp */
class exception : public std::runtime_error
{
	public :
		exception(int errorNumber, const std::string& msg) :
			std::runtime_error(msg), m_errno(errorNumber) {}
		~exception() throw () {}
		int errorNumber() const { return m_errno; }
	private :
		int m_errno;
};

namespace detail {

inline void
check(nemo_status_t status)
{
	if(status != NEMO_OK) {
		throw nemo::exception(status, nemo_strerror());
	}
}

inline const std::vector<synapse_id>&
copyIds(synapse_id* ids, size_t len, std::vector<synapse_id>& out)
{
	out.assign(ids, ids + len);
	return out;
}

} // namespace detail

/* src/nemo/ReadableNetwork.hpp */
class ReadableNetwork
{
	public :
		virtual ~ReadableNetwork() { }
		unsigned getSynapseSource(const synapse_id& id) const { return unsigned(id >> 32); }
		virtual unsigned getSynapseTarget(const synapse_id&) const = 0;
		virtual unsigned getSynapseDelay(const synapse_id&) const = 0;
		virtual float getSynapseWeight(const synapse_id&) const = 0;
		virtual unsigned char getSynapsePlastic(const synapse_id&) const = 0;
		virtual const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron) = 0;
};

class Simulation;

/* src/nemo/Network.hpp */
class Network : public ReadableNetwork
{
	public :
		Network() : m_h(nemo_new_network()) {
			if(!m_h) throw nemo::exception(NEMO_ALLOCATION_ERROR, nemo_strerror());
		}
		~Network() { nemo_delete_network(m_h); }

		unsigned addNeuronType(const std::string& name) {
			unsigned t = 0;
			detail::check(nemo_add_neuron_type(m_h, name.c_str(), &t));
			return t;
		}
		void addNeuron(unsigned type, unsigned idx, unsigned nargs, const float args[]) {
			detail::check(nemo_add_neuron(m_h, type, idx, nargs, const_cast<float*>(args)));
		}
		void addNeuron(unsigned idx, float a, float b, float c, float d, float u, float v, float sigma) {
			detail::check(nemo_add_neuron_iz(m_h, idx, a, b, c, d, u, v, sigma));
		}
		void setNeuron(unsigned idx, unsigned nargs, const float args[]) {
			detail::check(nemo_set_neuron_n(m_h, idx, nargs, const_cast<float*>(args)));
		}
		void setNeuron(unsigned idx, float a, float b, float c, float d, float u, float v, float sigma) {
			detail::check(nemo_set_neuron_iz_n(m_h, idx, a, b, c, d, u, v, sigma));
		}
		synapse_id addSynapse(unsigned source, unsigned target, unsigned delay, float weight,
				unsigned char plastic) {
			synapse_id id = 0;
			detail::check(nemo_add_synapse(m_h, source, target, delay, weight, plastic, &id));
			return id;
		}

		float getNeuronParameter(unsigned neuron, unsigned parameter) const {
			float x = 0;
			detail::check(nemo_get_neuron_parameter_n(m_h, neuron, parameter, &x));
			return x;
		}
		float getNeuronState(unsigned neuron, unsigned var) const {
			float x = 0;
			detail::check(nemo_get_neuron_state_n(m_h, neuron, var, &x));
			return x;
		}
		void setNeuronParameter(unsigned neuron, unsigned parameter, float value) {
			detail::check(nemo_set_neuron_parameter_n(m_h, neuron, parameter, value));
		}
		void setNeuronState(unsigned neuron, unsigned var, float value) {
			detail::check(nemo_set_neuron_state_n(m_h, neuron, var, value));
		}

		unsigned getSynapseTarget(const synapse_id& id) const {
			unsigned x = 0;
			detail::check(nemo_get_synapse_target_n(m_h, id, &x));
			return x;
		}
		unsigned getSynapseDelay(const synapse_id& id) const {
			unsigned x = 0;
			detail::check(nemo_get_synapse_delay_n(m_h, id, &x));
			return x;
		}
		float getSynapseWeight(const synapse_id& id) const {
			float x = 0;
			detail::check(nemo_get_synapse_weight_n(m_h, id, &x));
			return x;
		}
		unsigned char getSynapsePlastic(const synapse_id& id) const {
			unsigned char x = 0;
			detail::check(nemo_get_synapse_plastic_n(m_h, id, &x));
			return x;
		}
		const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron) {
			synapse_id* ids = NULL;
			size_t len = 0;
			detail::check(nemo_get_synapses_from_n(m_h, neuron, &ids, &len));
			return detail::copyIds(ids, len, m_ids);
		}

		unsigned maxDelay() const {
			unsigned d = 0;
			float lo = 0, hi = 0;
			detail::check(nemo_b200_network_stats(m_h, &d, &lo, &hi));
			return d;
		}
		float maxWeight() const {
			unsigned d = 0;
			float lo = 0, hi = 0;
			detail::check(nemo_b200_network_stats(m_h, &d, &lo, &hi));
			return hi;
		}
		float minWeight() const {
			unsigned d = 0;
			float lo = 0, hi = 0;
			detail::check(nemo_b200_network_stats(m_h, &d, &lo, &hi));
			return lo;
		}
		unsigned neuronCount() const {
			unsigned n = 0;
			detail::check(nemo_neuron_count(m_h, &n));
			return n;
		}

		/* the C handle, for the extensions of include/nemo_b200.h */
		nemo_network_t handle() const { return m_h; }

	private :
		nemo_network_t m_h;
		std::vector<synapse_id> m_ids;
		Network(const Network&);
		Network& operator=(const Network&);
};

/* src/nemo/Configuration.hpp. The settings live in this object (so that it
 * copies) and are written into a C configuration when a simulation is made. */
class Configuration
{
	public :
		Configuration() :
			m_logging(false), m_partitionSize(0), m_stdp(false), m_minE(0), m_maxE(0), m_minI(0),
			m_maxI(0), m_writeOnly(false), m_cpu(false), m_device(-1), m_stdpEnabled(false),
			m_stdpPeriod(0), m_stdpReward(0) {}

		void enableLogging() { m_logging = true; }
		void disableLogging() { m_logging = false; }
		bool loggingEnabled() const { return m_logging; }

		void setCudaPartitionSize(unsigned ps) { m_partitionSize = ps; }
		unsigned cudaPartitionSize() const { return m_partitionSize; }

		/* excitatory weights in [0, maxWeight], inhibitory in [minWeight, 0]
		 * (src/nemo/Configuration.cpp:148-151) */
		void setStdpFunction(const std::vector<float>& prefire, const std::vector<float>& postfire,
				float minWeight, float maxWeight) {
			setStdpFunction(prefire, postfire, 0, maxWeight, 0, minWeight);
		}
		void setStdpFunction(const std::vector<float>& prefire, const std::vector<float>& postfire,
				float minExcitatoryWeight, float maxExcitatoryWeight,
				float minInhibitoryWeight, float maxInhibitoryWeight) {
			/* validated now, as the reference does */
			nemo_configuration_t c = nemo_new_configuration();
			if(!c) throw nemo::exception(NEMO_ALLOCATION_ERROR, nemo_strerror());
			const nemo_status_t s = nemo_set_stdp_function(c,
					const_cast<float*>(prefire.empty() ? NULL : &prefire[0]), prefire.size(),
					const_cast<float*>(postfire.empty() ? NULL : &postfire[0]), postfire.size(),
					minExcitatoryWeight, maxExcitatoryWeight, minInhibitoryWeight, maxInhibitoryWeight);
			nemo_delete_configuration(c);
			detail::check(s);
			m_stdp = true;
			m_prefire = prefire;
			m_postfire = postfire;
			m_minE = minExcitatoryWeight;
			m_maxE = maxExcitatoryWeight;
			m_minI = minInhibitoryWeight;
			m_maxI = maxInhibitoryWeight;
		}

		void setWriteOnlySynapses() { m_writeOnly = true; }
		bool writeOnlySynapses() const { return m_writeOnly; }

		void setCudaBackend(int device = -1) { m_cpu = false; m_device = device; }
		void setCpuBackend() {
			throw nemo::exception(NEMO_API_UNSUPPORTED, "The B200 library has no CPU backend");
		}
		backend_t backend() const { return m_cpu ? NEMO_BACKEND_CPU : NEMO_BACKEND_CUDA; }
		int cudaDevice() const { return m_device; }

		bool stdpEnabled() const { return m_stdpEnabled; }
		void setStdpEnabled(bool isEnabled) { m_stdpEnabled = isEnabled; }
		void setStdpPeriod(unsigned period) { m_stdpPeriod = period; }
		unsigned stdpPeriod() const { return m_stdpPeriod; }
		void setStdpReward(float reward) { m_stdpReward = reward; }
		float stdpReward() const { return m_stdpReward; }
		void setStdpParams(unsigned period, float reward) {
			m_stdpEnabled = true;
			m_stdpPeriod = period;
			m_stdpReward = reward;
		}

		const char* backendDescription() const {
			nemo_configuration_t c = make();
			const char* d = NULL;
			const nemo_status_t s = nemo_backend_description(c, &d);
			m_description = (s == NEMO_OK && d) ? d : "";
			nemo_delete_configuration(c);
			detail::check(s);
			return m_description.c_str();
		}

		/* a C configuration with these settings (the caller deletes it) */
		nemo_configuration_t make() const {
			nemo_configuration_t c = nemo_new_configuration();
			if(!c) throw nemo::exception(NEMO_ALLOCATION_ERROR, nemo_strerror());
			nemo_status_t s = NEMO_OK;
			if(m_logging) s = nemo_log_stdout(c);
			if(s == NEMO_OK && m_stdp) {
				s = nemo_set_stdp_function(c,
						const_cast<float*>(m_prefire.empty() ? NULL : &m_prefire[0]), m_prefire.size(),
						const_cast<float*>(m_postfire.empty() ? NULL : &m_postfire[0]), m_postfire.size(),
						m_minE, m_maxE, m_minI, m_maxI);
			}
			if(s == NEMO_OK && m_writeOnly) s = nemo_set_write_only_synapses(c);
			if(s == NEMO_OK) s = nemo_set_cuda_backend(c, m_device);
			if(s != NEMO_OK) {
				nemo_delete_configuration(c);
				detail::check(s);
			}
			return c;
		}

	private :
		bool m_logging;
		unsigned m_partitionSize;
		bool m_stdp;
		std::vector<float> m_prefire, m_postfire;
		float m_minE, m_maxE, m_minI, m_maxI;
		bool m_writeOnly;
		bool m_cpu;
		int m_device;
		bool m_stdpEnabled;
		unsigned m_stdpPeriod;
		float m_stdpReward;
		mutable std::string m_description;
};

/* src/nemo/Simulation.hpp; made by nemo::simulation() */
class Simulation : public ReadableNetwork
{
	public :
		typedef std::vector<unsigned> firing_output;
		typedef std::vector<unsigned> firing_stimulus;
		typedef std::vector< std::pair<unsigned, float> > current_stimulus;

		explicit Simulation(nemo_simulation_t h) : m_h(h) {}
		virtual ~Simulation() { nemo_delete_simulation(m_h); }

		virtual const firing_output& step() {
			return step(firing_stimulus(), current_stimulus());
		}
		virtual const firing_output& step(const firing_stimulus& fstim) {
			return step(fstim, current_stimulus());
		}
		virtual const firing_output& step(const current_stimulus& istim) {
			return step(firing_stimulus(), istim);
		}
		virtual const firing_output& step(const firing_stimulus& fstim, const current_stimulus& istim) {
			m_inidx.resize(istim.size());
			m_icur.resize(istim.size());
			for(size_t k = 0; k < istim.size(); ++k) {
				m_inidx[k] = istim[k].first;
				m_icur[k] = istim[k].second;
			}
			unsigned* fired = NULL;
			size_t nfired = 0;
			detail::check(nemo_step(m_h,
					const_cast<unsigned*>(fstim.empty() ? NULL : &fstim[0]), fstim.size(),
					m_inidx.empty() ? NULL : &m_inidx[0], m_icur.empty() ? NULL : &m_icur[0], istim.size(),
					&fired, &nfired));
			m_fired.assign(fired, fired + nfired);
			return m_fired;
		}

		virtual void setNeuron(unsigned idx, unsigned nargs, const float args[]) {
			detail::check(nemo_set_neuron_s(m_h, idx, nargs, const_cast<float*>(args)));
		}
		void setNeuron(unsigned idx, float a, float b, float c, float d, float u, float v, float sigma) {
			detail::check(nemo_set_neuron_iz_s(m_h, idx, a, b, c, d, u, v, sigma));
		}
		virtual void setNeuronState(unsigned neuron, unsigned var, float value) {
			detail::check(nemo_set_neuron_state_s(m_h, neuron, var, value));
		}
		virtual void setNeuronParameter(unsigned neuron, unsigned parameter, float value) {
			detail::check(nemo_set_neuron_parameter_s(m_h, neuron, parameter, value));
		}
		virtual void applyStdp(float reward) {
			detail::check(nemo_apply_stdp(m_h, reward));
		}
		virtual float getNeuronState(unsigned neuron, unsigned var) const {
			float x = 0;
			detail::check(nemo_get_neuron_state_s(m_h, neuron, var, &x));
			return x;
		}
		virtual float getNeuronParameter(unsigned neuron, unsigned parameter) const {
			float x = 0;
			detail::check(nemo_get_neuron_parameter_s(m_h, neuron, parameter, &x));
			return x;
		}
		virtual float getMembranePotential(unsigned neuron) const {
			float x = 0;
			detail::check(nemo_get_membrane_potential(m_h, neuron, &x));
			return x;
		}
		virtual unsigned getSynapseTarget(const synapse_id& id) const {
			unsigned x = 0;
			detail::check(nemo_get_synapse_target_s(m_h, id, &x));
			return x;
		}
		virtual unsigned getSynapseDelay(const synapse_id& id) const {
			unsigned x = 0;
			detail::check(nemo_get_synapse_delay_s(m_h, id, &x));
			return x;
		}
		virtual float getSynapseWeight(const synapse_id& id) const {
			float x = 0;
			detail::check(nemo_get_synapse_weight_s(m_h, id, &x));
			return x;
		}
		virtual unsigned char getSynapsePlastic(const synapse_id& id) const {
			unsigned char x = 0;
			detail::check(nemo_get_synapse_plastic_s(m_h, id, &x));
			return x;
		}
		virtual const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron) {
			synapse_id* ids = NULL;
			size_t len = 0;
			detail::check(nemo_get_synapses_from_s(m_h, neuron, &ids, &len));
			return detail::copyIds(ids, len, m_ids);
		}
		virtual unsigned long elapsedWallclock() const {
			unsigned long x = 0;
			detail::check(nemo_elapsed_wallclock(m_h, &x));
			return x;
		}
		virtual unsigned long elapsedSimulation() const {
			unsigned long x = 0;
			detail::check(nemo_elapsed_simulation(m_h, &x));
			return x;
		}
		virtual void resetTimer() {
			detail::check(nemo_reset_timer(m_h));
		}

		/* the C handle, for the extensions of include/nemo_b200.h */
		nemo_simulation_t handle() const { return m_h; }

	private :
		nemo_simulation_t m_h;
		firing_output m_fired;
		std::vector<unsigned> m_inidx;
		std::vector<float> m_icur;
		std::vector<synapse_id> m_ids;
		Simulation(const Simulation&);
		Simulation& operator=(const Simulation&);
};

/* src/nemo.hpp: a simulation of the network on the configured device. The
 * reference returns NULL when no backend can be made; this throws
 * nemo::exception with the reason instead, so that the caller sees it. The
 * caller deletes the simulation. */
inline Simulation*
simulation(const Network& net, const Configuration& conf)
{
	nemo_configuration_t c = conf.make();
	nemo_simulation_t s = nemo_new_simulation(net.handle(), c);
	nemo_delete_configuration(c);
	if(!s) {
		throw nemo::exception(nemo_b200_last_status(), nemo_strerror());
	}
	return new Simulation(s);
}

inline unsigned
cudaDeviceCount()
{
	unsigned n = 0;
	detail::check(nemo_cuda_device_count(&n));
	return n;
}

inline const char*
cudaDeviceDescription(unsigned device)
{
	const char* d = NULL;
	detail::check(nemo_cuda_device_description(device, &d));
	return d;
}

inline const char* version() { return nemo_version(); }

inline void addPluginPath(const std::string& dir) { detail::check(nemo_add_plugin_path(dir.c_str())); }

} // namespace nemo

#endif
