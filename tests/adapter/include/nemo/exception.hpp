/* Stand-in for src/nemo/exception.hpp: an error with a status code. */
#ifndef NEMO_EXCEPTION_HPP
#define NEMO_EXCEPTION_HPP
#include <stdexcept>
#include <string>
#include <nemo/types.h>
namespace nemo {
class exception : public std::runtime_error
{
	public :
		exception(int errorNumber, const std::string& msg) : std::runtime_error(msg), m_errno(errorNumber) {}
		int errorNumber() const { return m_errno; }
	private :
		int m_errno;
};
}
#endif
