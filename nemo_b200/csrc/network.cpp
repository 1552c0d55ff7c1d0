/* Network, configuration and neuron-type descriptors (see network.hpp). */

#include "network.hpp"

#include <dlfcn.h>
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

namespace nemo_b200 {

/* ---------------- neuron-type descriptors ---------------- */

static std::vector<std::string> g_extraPaths;
static std::mutex g_pathLock;

static bool
isDir(const std::string& p)
{
	struct stat st;
	return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

static bool
isFile(const std::string& p)
{
	struct stat st;
	return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

/* src/nemo/Plugin.cpp:186-200: paths added later are searched first */
void
addPluginPath(const std::string& dir)
{
	if(!isDir(dir)) {
		fail(NEMO_INVALID_INPUT, "Plugin path does not exist: " + dir);
	}
	std::lock_guard<std::mutex> g(g_pathLock);
	g_extraPaths.insert(g_extraPaths.begin(), dir);
}

/* The directory of the .ini descriptors shipped with this library:
 * <directory of libnemo_b200.so>/plugins */
static std::string
systemPluginDir()
{
	Dl_info info;
	if(dladdr((void*) &systemPluginDir, &info) && info.dli_fname) {
		std::string lib = info.dli_fname;
		size_t slash = lib.rfind('/');
		return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/plugins";
	}
	return "plugins";
}

/* src/nemo/NeuronType.cpp:40-72: extra paths, then ~/.nemo/plugins, then the
 * system directory */
static std::string
configurationFile(const std::string& name)
{
	std::vector<std::string> dirs;
	{
		std::lock_guard<std::mutex> g(g_pathLock);
		dirs = g_extraPaths;
	}
	if(const char* home = getenv("HOME")) {
		dirs.push_back(std::string(home) + "/.nemo/plugins");
	}
	dirs.push_back(systemPluginDir());
	for(const std::string& d : dirs) {
		std::string p = d + "/" + name + ".ini";
		if(isFile(p)) {
			return p;
		}
	}
	fail(NEMO_INVALID_INPUT, "Could not find .ini file for plugin " + name);
}

static std::string
trim(const std::string& s)
{
	size_t b = s.find_first_not_of(" \t\r\n");
	if(b == std::string::npos) return "";
	size_t e = s.find_last_not_of(" \t\r\n");
	return s.substr(b, e - b + 1);
}

static bool
parseBool(const std::string& v, const std::string& key, const std::string& file)
{
	std::string l = v;
	std::transform(l.begin(), l.end(), l.begin(), ::tolower);
	if(l == "true" || l == "1" || l == "yes" || l == "on") return true;
	if(l == "false" || l == "0" || l == "no" || l == "off") return false;
	fail(NEMO_INVALID_INPUT, "Error parsing neuron model configuration file " + file
			+ ": invalid boolean '" + v + "' for " + key);
}

static unsigned
parseUnsigned(const std::string& v, const std::string& key, const std::string& file)
{
	char* end = nullptr;
	unsigned long x = strtoul(v.c_str(), &end, 10);
	if(v.empty() || *end != '\0' || v[0] == '-') {
		fail(NEMO_INVALID_INPUT, "Error parsing neuron model configuration file " + file
				+ ": invalid value '" + v + "' for " + key);
	}
	return unsigned(x);
}

static ModelKind
modelKind(const std::string& name)
{
	static const std::map<std::string, ModelKind> kinds = {
		{"Izhikevich", MODEL_IZHIKEVICH}, {"IF_curr_exp", MODEL_IF_CURR_EXP},
		{"QIF", MODEL_QIF}, {"HH", MODEL_HH},
		{"PoissonSource", MODEL_POISSON_SOURCE}, {"Input", MODEL_INPUT}};
	auto it = kinds.find(name);
	return it == kinds.end() ? MODEL_COUNT : it->second;
}

/* src/nemo/NeuronType.cpp:94-158. INI syntax: "key=value", "[section]"
 * prefixes following keys with "section.", '#' starts a comment; unknown
 * keys are ignored. */
NeuronType
loadNeuronType(const std::string& name)
{
	std::string file = configurationFile(name);
	std::ifstream in(file);
	if(!in) {
		fail(NEMO_IO_ERROR, "Failed to open neuron model configuration file " + file + ": " + strerror(errno));
	}
	std::map<std::string, std::string> kv;
	std::string section, line;
	while(std::getline(in, line)) {
		size_t hash = line.find('#');
		if(hash != std::string::npos) line = line.substr(0, hash);
		line = trim(line);
		if(line.empty()) continue;
		if(line.front() == '[' && line.back() == ']') {
			section = trim(line.substr(1, line.size() - 2));
			continue;
		}
		size_t eq = line.find('=');
		if(eq == std::string::npos) {
			fail(NEMO_INVALID_INPUT, "Error parsing neuron model configuration file " + file + ": " + line);
		}
		std::string key = trim(line.substr(0, eq));
		kv[section.empty() ? key : section + "." + key] = trim(line.substr(eq + 1));
	}
	auto required = [&](const char* key) -> const std::string& {
		auto it = kv.find(key);
		if(it == kv.end()) {
			fail(NEMO_INVALID_INPUT, std::string("Missing parameter '") + key + "' in configuration file " + file);
		}
		return it->second;
	};
	auto optBool = [&](const char* key, bool def) {
		auto it = kv.find(key);
		return it == kv.end() ? def : parseBool(it->second, key, file);
	};
	NeuronType t;
	t.name = name;
	t.nParam = parseUnsigned(required("parameters"), "parameters", file);
	t.nState = parseUnsigned(required("state-variables"), "state-variables", file);
	t.membranePotential = parseUnsigned(required("membrane-potential"), "membrane-potential", file);
	t.nrand = parseBool(required("rng.normal"), "rng.normal", file);
	t.rcmSources = optBool("rcm.sources", false);
	t.rcmDelays = optBool("rcm.delays", false);
	t.rcmForward = optBool("rcm.forward", false);
	t.rcmWeights = optBool("rcm.weights", false);
	t.backendCpu = optBool("backends.cpu", false);
	t.backendCuda = optBool("backends.cuda", false);
	auto h = kv.find("history");
	t.history = h == kv.end() ? 1 : parseUnsigned(h->second, "history", file);
	t.pluginDir = file.substr(0, file.rfind('/'));
	t.kind = modelKind(name);
	if(t.kind == MODEL_COUNT) {
		/* not a built-in model: a GPU plugin beside the .ini, as the
		 * reference keeps lib<name>.so in <dir>/{cpu,cuda}/ */
		const std::string lib = t.pluginDir + "/b200/lib" + name + ".so";
		if(isFile(lib)) {
			t.kind = MODEL_EXTERNAL;
			t.b200Plugin = lib;
		}
	}
	return t;
}

/* ---------------- STDP function (src/nemo/StdpFunction.cpp:9-107) ---------------- */

StdpFunction::StdpFunction(const std::vector<float>& pre, const std::vector<float>& post,
		float minE, float maxE, float minI, float maxI) :
	prefire(pre), postfire(post), minE(minE), maxE(maxE), minI(minI), maxI(maxI)
{
	if(maxI > 0.0f || minI > 0.0f) {
		fail(NEMO_INVALID_INPUT, "STDP function should not have positive limits for inhibitory synapses");
	}
	if(maxE < 0.0f || minE < 0.0f) {
		fail(NEMO_INVALID_INPUT, "STDP function should not have negative limits for excitatory synapses");
	}
	if(maxE < minE) {
		fail(NEMO_INVALID_INPUT, "STDP should have maximum excitatory weight >= minimum excitatory weight");
	}
	if(maxI > minI) {
		fail(NEMO_INVALID_INPUT, "STDP should have abs(maximum inhibitory weight) >= abs(minimum inhibitory weight)");
	}
	if(prefire.size() + postfire.size() > 64) {
		fail(NEMO_INVALID_INPUT, "size of STDP window too large");
	}
}

void
StdpFunction::verifyDynamicWindowLength(unsigned dmax) const
{
	if(dmax + postfire.size() > 64) {
		fail(NEMO_INVALID_INPUT, "Max delay + postfire part of STDP function must be <= 64");
	}
}

/* Bit n of the window mask: the postfire part from its far end, then the
 * prefire part (StdpFunction.cpp:51-68); bit 0 is the end of the window. */
static uint64_t
windowBits(const StdpFunction& f, bool positive)
{
	uint64_t bits = 0;
	unsigned n = 0;
	for(auto it = f.postfire.rbegin(); it != f.postfire.rend(); ++it, ++n) {
		if(positive ? *it > 0.0f : *it < 0.0f) bits |= uint64_t(1) << n;
	}
	for(float x : f.prefire) {
		if(positive ? x > 0.0f : x < 0.0f) bits |= uint64_t(1) << n;
		n++;
	}
	return bits;
}

uint64_t StdpFunction::potentiationBits() const { return windowBits(*this, true); }
uint64_t StdpFunction::depressionBits() const { return windowBits(*this, false); }

/* ---------------- network ---------------- */

/* src/nemo/NetworkImpl.cpp:428-438 */
unsigned
Network::addNeuronType(const std::string& name)
{
	auto it = typeIds.find(name);
	if(it != typeIds.end()) {
		return it->second;
	}
	NeuronGroup g;
	g.type = loadNeuronType(name);
	g.param.resize(g.type.nParam);
	g.state.resize(g.type.nState);
	unsigned id = unsigned(groups.size());
	groups.push_back(std::move(g));
	typeIds[name] = id;
	return id;
}

static std::string
argCountMessage(const char* what, unsigned expected, unsigned found)
{
	std::ostringstream msg;
	msg << "Unexpected number of parameters/state variables when " << what
		<< " neuron. Expected " << expected << ", found " << found;
	return msg.str();
}

/* src/nemo/NetworkImpl.cpp:471-476, Neurons.cpp:29-48. The neuron joins its
 * type before the duplicate check, as in the reference, so a rejected
 * duplicate later also fails simulation construction. */
void
Network::addNeuron(unsigned type, unsigned gidx, unsigned nargs, const float* args)
{
	if(type >= groups.size()) {
		fail(NEMO_INVALID_INPUT, "Invalid neuron type id " + std::to_string(type));
	}
	NeuronGroup& g = groups[type];
	if(nargs != g.type.nParam + g.type.nState) {
		fail(NEMO_INVALID_INPUT, argCountMessage("adding", g.type.nParam + g.type.nState, nargs));
	}
	for(unsigned i = 0; i < g.type.nParam; ++i) g.param[i].push_back(*args++);
	for(unsigned i = 0; i < g.type.nState; ++i) g.state[i].push_back(*args++);
	g.gidx.push_back(gidx);
	if(!mapper.emplace(gidx, std::make_pair(type, uint32_t(g.gidx.size() - 1))).second) {
		fail(NEMO_INVALID_INPUT, "Duplicate neuron index " + std::to_string(gidx));
	}
}

std::pair<uint32_t, uint32_t>
Network::address(unsigned gidx) const
{
	auto it = mapper.find(gidx);
	if(it == mapper.end()) {
		fail(NEMO_INVALID_INPUT, "Non-existing neuron index " + std::to_string(gidx));
	}
	return it->second;
}

void
Network::setNeuron(unsigned gidx, unsigned nargs, const float* args)
{
	auto a = address(gidx);
	NeuronGroup& g = groups[a.first];
	if(nargs != g.type.nParam + g.type.nState) {
		fail(NEMO_INVALID_INPUT, argCountMessage("modifying", g.type.nParam + g.type.nState, nargs));
	}
	for(unsigned i = 0; i < g.type.nParam; ++i) g.param[i][a.second] = *args++;
	for(unsigned i = 0; i < g.type.nState; ++i) g.state[i][a.second] = *args++;
}

static void
checkIndex(unsigned i, unsigned n, const char* what)
{
	if(i >= n) {
		fail(NEMO_INVALID_INPUT, std::string("Invalid ") + what + " index " + std::to_string(i));
	}
}

float
Network::getNeuronState(unsigned gidx, unsigned var) const
{
	auto a = address(gidx);
	checkIndex(var, groups[a.first].type.nState, "state variable");
	return groups[a.first].state[var][a.second];
}

float
Network::getNeuronParameter(unsigned gidx, unsigned param) const
{
	auto a = address(gidx);
	checkIndex(param, groups[a.first].type.nParam, "parameter");
	return groups[a.first].param[param][a.second];
}

void
Network::setNeuronState(unsigned gidx, unsigned var, float val)
{
	auto a = address(gidx);
	checkIndex(var, groups[a.first].type.nState, "state variable");
	groups[a.first].state[var][a.second] = val;
}

void
Network::setNeuronParameter(unsigned gidx, unsigned param, float val)
{
	auto a = address(gidx);
	checkIndex(param, groups[a.first].type.nParam, "parameter");
	groups[a.first].param[param][a.second] = val;
}

/* src/nemo/NetworkImpl.cpp:492-511 */
synapse_id
Network::addSynapse(unsigned source, unsigned target, unsigned delay, float weight, unsigned char pl)
{
	if(delay < 1) {
		fail(NEMO_INVALID_INPUT, "Invalid delay (" + std::to_string(delay) + ") for synapse between "
				+ std::to_string(source) + " and " + std::to_string(target));
	}
	if(source != m_lastSrc || m_lastCount == nullptr) {
		m_lastCount = &m_srcCount[source];
		m_lastSrc = source;
	}
	uint32_t id = (*m_lastCount)++;
	src.push_back(source);
	tgt.push_back(target);
	dly.push_back(delay);
	wgt.push_back(weight);
	plastic.push_back(pl != 0);
	sid.push_back(id);
	m_maxDelay = std::max(m_maxDelay, delay);
	m_indexed = false;
	return (uint64_t(source) << 32) | uint64_t(id);
}

void
Network::indexBySource() const
{
	if(m_indexed) return;
	m_srcRange.clear();
	size_t offset = 0;
	for(const auto& kv : m_srcCount) {
		m_srcRange[kv.first] = std::make_pair(offset, 0u);
		offset += kv.second;
	}
	m_bySource.assign(src.size(), 0);
	for(size_t i = 0; i < src.size(); ++i) {
		auto& r = m_srcRange[src[i]];
		m_bySource[r.first + r.second++] = i;
	}
	m_indexed = true;
}

/* position of a synapse in the insertion-order arrays; out-of-range ids raise
 * std::out_of_range like the reference's vector::at (NEMO_UNKNOWN_ERROR) */
size_t
Network::synapsePosition(synapse_id id) const
{
	indexBySource();
	uint32_t source = uint32_t(id >> 32);
	auto it = m_srcRange.find(source);
	if(it == m_srcRange.end()) {
		fail(NEMO_INVALID_INPUT, "synapses of non-existing neuron (" + std::to_string(source) + ") requested");
	}
	uint32_t i = uint32_t(id & 0xffffffffu);
	if(i >= it->second.second) {
		throw std::out_of_range("synapse id out of range");
	}
	return m_bySource[it->second.first + i];
}

const std::vector<synapse_id>&
Network::getSynapsesFrom(unsigned source)
{
	m_queried.clear();
	auto it = m_srcCount.find(source);
	if(it != m_srcCount.end()) {
		m_queried.resize(it->second);
		for(uint32_t i = 0; i < it->second; ++i) {
			m_queried[i] = (uint64_t(source) << 32) | i;
		}
	}
	return m_queried;
}

/* Instances in order; a type takes the merged group of its name, in order of
 * first appearance, so each instance keeps its own type order and neuron
 * order within its neurons. */
Network
Network::merge(const std::vector<const Network*>& nets, std::vector<uint32_t>* base)
{
	Network m;
	base->assign(nets.size() + 1, 0u);
	uint64_t next = 0;
	for(size_t j = 0; j < nets.size(); ++j) {
		const Network& n = *nets[j];
		(*base)[j] = uint32_t(next);
		uint64_t span = 0;
		for(const NeuronGroup& g : n.groups) {
			for(uint32_t gi : g.gidx) span = std::max<uint64_t>(span, uint64_t(gi) + 1);
		}
		if(next + span >= (uint64_t(1) << 32)) {
			fail(NEMO_INVALID_INPUT, "Batch: the networks' neuron indices do not fit in 32 bits together");
		}
		const uint32_t off = uint32_t(next);
		uint32_t local = 0;
		for(const NeuronGroup& g : n.groups) {
			const unsigned t = m.addNeuronType(g.type.name);
			NeuronGroup& mg = m.groups[t];
			if(m.seedKey.size() < m.groups.size()) m.seedKey.resize(m.groups.size());
			for(unsigned p = 0; p < g.type.nParam; ++p) {
				mg.param[p].insert(mg.param[p].end(), g.param[p].begin(), g.param[p].end());
			}
			for(unsigned s = 0; s < g.type.nState; ++s) {
				mg.state[s].insert(mg.state[s].end(), g.state[s].begin(), g.state[s].end());
			}
			for(uint32_t gi : g.gidx) {
				mg.gidx.push_back(gi + off);
				m.seedKey[t].push_back((uint64_t(j) << 32) | local++);
			}
		}
		const size_t S = n.src.size();
		for(size_t k = 0; k < S; ++k) {
			m.src.push_back(n.src[k] + off);
			m.tgt.push_back(n.tgt[k] + off);
		}
		m.dly.insert(m.dly.end(), n.dly.begin(), n.dly.end());
		m.wgt.insert(m.wgt.end(), n.wgt.begin(), n.wgt.end());
		m.plastic.insert(m.plastic.end(), n.plastic.begin(), n.plastic.end());
		m.sid.insert(m.sid.end(), n.sid.begin(), n.sid.end());
		m.m_maxDelay = std::max(m.m_maxDelay, n.m_maxDelay);
		next += span;
	}
	(*base)[nets.size()] = uint32_t(next);
	return m;
}

Network
Network::subsetByTarget(const std::function<bool(uint32_t)>& keepTarget) const
{
	Network m;
	m.groups = groups;
	m.typeIds = typeIds;
	m.mapper = mapper;
	m.izType = izType;
	m.seedKey = seedKey;
	for(size_t k = 0; k < src.size(); ++k) {
		if(!keepTarget(tgt[k])) continue;
		m.src.push_back(src[k]);
		m.tgt.push_back(tgt[k]);
		m.dly.push_back(dly[k]);
		m.wgt.push_back(wgt[k]);
		m.plastic.push_back(plastic[k]);
		m.sid.push_back(sid[k]);
		m.m_srcCount[src[k]]++;
	}
	m.m_maxDelay = m_maxDelay;
	return m;
}

unsigned
Network::neuronCount() const
{
	size_t total = 0;
	for(const NeuronGroup& g : groups) total += g.gidx.size();
	return unsigned(total);
}

} // namespace nemo_b200
