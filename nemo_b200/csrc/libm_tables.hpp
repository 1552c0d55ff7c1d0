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

/* The inputs on which host glibc expf differs from the rounded device
 * candidate libm::exp_candidate_d (all finite floats in [-104, 89]; outside
 * that range both give 0 or infinity), sorted by input bits, with glibc's
 * results, and the largest libm::exp_midpoint_units of their candidates
 * (nearUnits; tau = nearUnits / 2^29 of the float spacing): an input whose
 * candidate lies farther from the rounding midpoint is never an exception. */
struct ExpExceptions {
	std::vector<uint32_t> keys;
	std::vector<uint32_t> values;
	uint32_t nearUnits = 0;
	double tau = 0.0;
	/* the same pairs as the device hash (libm::exp_lookup): 2^slotBits slots
	 * at most one third full, probe sequences of at most slotProbe slots */
	std::vector<uint64_t> slots;
	uint32_t slotBits = 0;
	uint32_t slotProbe = 0;
};

/* Process-wide table: loaded from the cache file or built (all cores). */
const ExpExceptions& expExceptions();

} // namespace nemo_b200

#endif
