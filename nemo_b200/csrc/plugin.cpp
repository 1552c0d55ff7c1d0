#include "plugin.hpp"

#include <dlfcn.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "common.hpp"

namespace nemo_b200 {

static std::mutex g_pluginLock;
static std::map<std::string, std::unique_ptr<B200Plugin>> g_plugins;

const B200Plugin&
loadB200Plugin(const std::string& path)
{
	std::lock_guard<std::mutex> g(g_pluginLock);
	auto it = g_plugins.find(path);
	if(it != g_plugins.end()) {
		return *it->second;
	}
	/* RTLD_LOCAL: the plugin's own CUDA runtime and symbols stay its own */
	void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
	if(h == nullptr) {
		const char* e = dlerror();
		fail(NEMO_DL_ERROR, "Failed to load neuron model plugin " + path + ": " + (e ? e : "unknown error"));
	}
	std::unique_ptr<B200Plugin> p(new B200Plugin);
	p->path = path;
	p->update = reinterpret_cast<b200_update_neurons_t*>(dlsym(h, "b200_update_neurons"));
	p->init = reinterpret_cast<b200_init_neurons_t*>(dlsym(h, "b200_init_neurons"));
	if(p->update == nullptr) {
		dlclose(h);
		fail(NEMO_INVALID_INPUT, "Neuron model plugin " + path + " does not export b200_update_neurons");
	}
	/* a plugin compiled against another layout of the batch would read
	 * the wrong fields */
	const unsigned* abi = reinterpret_cast<const unsigned*>(dlsym(h, "b200_plugin_abi_version"));
	if(abi == nullptr || *abi != NEMO_B200_PLUGIN_ABI_VERSION) {
		const std::string got = abi == nullptr ? std::string("no b200_plugin_abi_version") : std::to_string(*abi);
		dlclose(h);
		fail(NEMO_DL_ERROR, "Neuron model plugin " + path + " was built for plugin ABI version " + got
				+ "; this library expects version " + std::to_string(NEMO_B200_PLUGIN_ABI_VERSION)
				+ " (rebuild it against include/nemo_b200_plugin.h)");
	}
	const B200Plugin& ref = *p;
	g_plugins.emplace(path, std::move(p));
	return ref;
}

} // namespace nemo_b200
