#ifndef NEMO_B200_LIBM_TABLES_HPP
#define NEMO_B200_LIBM_TABLES_HPP

#include <cstdint>
#include <string>
#include <vector>

namespace nemo_b200 {

/* 2-bit correction codes, 16 per word, indexed by libm::libm_index(float(u)) */
struct LibmTables {
	std::vector<uint32_t> sinCodes;
	std::vector<uint32_t> logCodes;
};

/* Process-wide tables: loaded from the cache file or built (all cores). */
const LibmTables& libmTables();

/* Always rebuilds (no cache); used by tests and the cache generator. */
LibmTables buildLibmTables();

std::string libmCachePath();

} // namespace nemo_b200

#endif
