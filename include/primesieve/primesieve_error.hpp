/// primesieve_error.hpp -- exception type of the primesieve-compatible C++ API
/// (reference include/primesieve/primesieve_error.hpp).
#ifndef PRIMESIEVE_ERROR_HPP
#define PRIMESIEVE_ERROR_HPP

#include <stdexcept>
#include <string>

namespace primesieve {

class primesieve_error : public std::runtime_error {
public:
  explicit primesieve_error(const std::string& msg) : std::runtime_error(msg) {}
};

} // namespace primesieve

#endif
