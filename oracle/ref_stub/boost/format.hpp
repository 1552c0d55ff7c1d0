/* ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * Stand-in for boost/format.hpp, enough to compile the reference's
 * src/nemo/StdpFunction.cpp without Boost: the reference uses boost::format
 * only to build the text of one error message
 * (StdpFunction::verifyDynamicWindowLength). This keeps the format string
 * and appends the arguments after it; no arithmetic depends on it. */
#ifndef ORACLE_REF_STUB_BOOST_FORMAT_HPP
#define ORACLE_REF_STUB_BOOST_FORMAT_HPP

#include <sstream>
#include <string>

namespace boost {

class format {
public:
	explicit format(const char* f) { m_text << f; }
	template<class T> format& operator%(const T& x) { m_text << " " << x; return *this; }
	std::string str() const { return m_text.str(); }
private:
	std::ostringstream m_text;
};

inline std::string str(const format& f) { return f.str(); }

} // namespace boost

#endif
