#ifndef NEMO_B200_COMMON_HPP
#define NEMO_B200_COMMON_HPP

/* Errors and small helpers shared by the host side of libnemo_b200. */

#include <cstdint>
#include <stdexcept>
#include <string>

#include <nemo/types.h>

namespace nemo_b200 {

/* Error carrying a NeMo status code (the role of nemo::exception,
 * src/nemo/exception.hpp:10-30). The C ABI reports code and message. */
class Exception : public std::runtime_error {
public:
	Exception(int code, const std::string& msg) : std::runtime_error(msg), m_code(code) {}
	int code() const { return m_code; }
private:
	int m_code;
};

[[noreturn]] void fail(int code, const std::string& msg);

/* Raise NEMO_CUDA_* on a failed CUDA runtime call. */
void cudaCheck(int err, const char* what, const char* file, int line);
#define NEMO_CUDA(call) ::nemo_b200::cudaCheck(int(call), #call, __FILE__, __LINE__)

inline uint64_t roundUp(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

} // namespace nemo_b200

#endif
