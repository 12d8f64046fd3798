/* Minimal stand-in for boost::lexical_cast, written for the reference-oracle
 * build only (Boost is not installed here). Converts through a stringstream,
 * which is what the reference relies on for integer <-> string casts. */
#ifndef MSG_SHIM_LEXICAL_CAST_HPP
#define MSG_SHIM_LEXICAL_CAST_HPP
#include <sstream>
#include <string>
#include <stdexcept>
namespace boost {
template <typename T, typename S>
T lexical_cast(const S& v) {
    std::stringstream ss;
    ss << v;
    T out;
    ss >> out;
    return out;
}
template <>
inline std::string lexical_cast<std::string, std::string>(const std::string& v) { return v; }
}  // namespace boost
#endif
