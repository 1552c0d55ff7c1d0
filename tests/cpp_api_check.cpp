// A C++ caller of the reference's API (nemo.hpp) built against this library:
// network construction and queries, configuration checks, and -- when run
// with "simulate" and a GPU -- a ring network simulated through
// nemo::simulation(). Prints "ok <what>" lines; exits non-zero on a failure.
#include <nemo.hpp>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#define EXPECT(cond) do { if(!(cond)) { std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #cond); return 1; } } while(0)

static int
construction()
{
	nemo::Network net;
	const unsigned iz = net.addNeuronType("Izhikevich");
	/* parameters a, b, c, d, sigma, then state u, v (Izhikevich.ini) */
	const float rs[7] = {0.02f, 0.2f, -65.0f, 8.0f, 0.0f, 0.2f * -65.0f, -65.0f};
	for(unsigned n = 0; n < 10; ++n) net.addNeuron(iz, n, 7, rs);
	net.addNeuron(10, 0.02f, 0.2f, -65.0f, 2.0f, -13.0f, -65.0f, 0.0f);
	EXPECT(net.neuronCount() == 11);
	const synapse_id a = net.addSynapse(0, 1, 3, 0.5f, 1);
	const synapse_id b = net.addSynapse(0, 2, 7, -1.25f, 0);
	net.addSynapse(4, 5, 1, 2.0f, 0);
	EXPECT((a >> 32) == 0 && (b >> 32) == 0 && a != b);
	EXPECT(net.getSynapseSource(b) == 0);
	EXPECT(net.getSynapseTarget(b) == 2 && net.getSynapseDelay(b) == 7);
	EXPECT(net.getSynapseWeight(a) == 0.5f && net.getSynapsePlastic(a) == 1);
	const std::vector<synapse_id>& from0 = net.getSynapsesFrom(0);
	EXPECT(from0.size() == 2 && from0[0] == a && from0[1] == b);
	EXPECT(net.maxDelay() == 7 && net.maxWeight() == 2.0f && net.minWeight() == -1.25f);
	EXPECT(net.getNeuronParameter(3, 0) == 0.02f && net.getNeuronState(3, 1) == -65.0f);
	net.setNeuronState(3, 1, -70.0f);
	EXPECT(net.getNeuronState(3, 1) == -70.0f);
	bool threw = false;
	try {
		net.addNeuron(iz, 3, 7, rs);   /* duplicate index */
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_INVALID_INPUT;
	}
	EXPECT(threw);
	std::printf("ok construction\n");
	return 0;
}

static int
configuration()
{
	nemo::Configuration conf;
	std::vector<float> pre(20, 0.1f), post(20, -0.12f);
	conf.setStdpFunction(pre, post, -1.0f, 1.0f);
	nemo::Configuration copy(conf);
	EXPECT(copy.backend() == NEMO_BACKEND_CUDA && copy.cudaDevice() == -1);
	std::vector<float> tooLong(50, 0.1f);
	bool threw = false;
	try {
		conf.setStdpFunction(tooLong, tooLong, 0.0f, 1.0f, 0.0f, -1.0f);   /* window > 64 */
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_INVALID_INPUT;
	}
	EXPECT(threw);
	threw = false;
	try {
		conf.setCpuBackend();
	} catch(nemo::exception& e) {
		threw = e.errorNumber() == NEMO_API_UNSUPPORTED;
	}
	EXPECT(threw);
	conf.setStdpParams(100, 1.0f);
	EXPECT(conf.stdpEnabled() && conf.stdpPeriod() == 100 && conf.stdpReward() == 1.0f);
	std::printf("ok configuration\n");
	return 0;
}

/* A ring of 64 Izhikevich neurons, delay 1 and a weight that makes every
 * spike fire the next neuron: neuron 0 forced at cycle 0, then neuron k fires
 * at cycle k (the reference's ring test, src/test). */
static int
ring()
{
	const unsigned N = 64;
	nemo::Network net;
	const unsigned iz = net.addNeuronType("Izhikevich");
	/* parameters a, b, c, d, sigma, then state u, v (Izhikevich.ini) */
	const float rs[7] = {0.02f, 0.2f, -65.0f, 8.0f, 0.0f, 0.2f * -65.0f, -65.0f};
	for(unsigned n = 0; n < N; ++n) {
		net.addNeuron(iz, n, 7, rs);
		net.addSynapse(n, (n + 1) % N, 1, 1000.0f, 0);
	}
	nemo::Configuration conf;
	nemo::Simulation* sim = nemo::simulation(net, conf);
	nemo::Simulation::firing_stimulus f(1, 0u);
	const nemo::Simulation::firing_output& fired0 = sim->step(f);
	EXPECT(fired0.size() == 1 && fired0[0] == 0);
	for(unsigned c = 1; c < 2 * N; ++c) {
		const nemo::Simulation::firing_output& fired = sim->step();
		EXPECT(fired.size() == 1 && fired[0] == c % N);
	}
	nemo::Simulation::current_stimulus istim;
	istim.push_back(std::make_pair(5u, 1.0f));
	sim->step(istim);
	EXPECT(sim->elapsedSimulation() == 2 * N + 1);
	EXPECT(std::isfinite(sim->getMembranePotential(5)));
	const std::vector<synapse_id>& from3 = sim->getSynapsesFrom(3);
	EXPECT(from3.size() == 1 && sim->getSynapseTarget(from3[0]) == 4 && sim->getSynapseWeight(from3[0]) == 1000.0f);
	delete sim;
	std::printf("ok ring\n");
	return 0;
}

int
main(int argc, char** argv)
{
	if(construction() || configuration()) return 1;
	if(argc > 1 && std::strcmp(argv[1], "simulate") == 0) {
		if(ring()) return 1;
	} else {
		/* without a device the simulation fails loudly, with a status */
		nemo::Network net;
		net.addNeuron(0, 0.02f, 0.2f, -65.0f, 8.0f, -13.0f, -65.0f, 0.0f);
		nemo::Configuration conf;
		bool threw = false;
		try {
			delete nemo::simulation(net, conf);
		} catch(nemo::exception& e) {
			threw = e.errorNumber() != NEMO_OK;
		}
		EXPECT(threw);
		std::printf("ok no device\n");
	}
	return 0;
}
