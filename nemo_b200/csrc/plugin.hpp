#ifndef NEMO_B200_PLUGIN_HPP
#define NEMO_B200_PLUGIN_HPP

/* Loading of GPU neuron-model plugins (include/nemo_b200_plugin.h): the
 * role of the reference's plugin loader (src/nemo/Plugin.cpp,
 * src/nemo/cpu/Neurons.cpp:19-20), for the B200 backend's signature. */

#include <string>

/* the library reads plugins' layout version; it defines none of its own */
#define NEMO_B200_PLUGIN_HOST
#include <nemo_b200_plugin.h>

namespace nemo_b200 {

struct B200Plugin {
	std::string path;
	b200_update_neurons_t* update = nullptr;
	b200_init_neurons_t* init = nullptr;   /* optional */
};

/* The plugin at `path`, opened once per process and kept open. Fails with
 * NEMO_DL_ERROR when it cannot be opened, NEMO_INVALID_INPUT when it does
 * not export b200_update_neurons, and NEMO_DL_ERROR when its
 * b200_plugin_abi_version is missing or is not NEMO_B200_PLUGIN_ABI_VERSION
 * (a plugin compiled against another layout of b200_neuron_batch). */
const B200Plugin& loadB200Plugin(const std::string& path);

} // namespace nemo_b200

#endif
