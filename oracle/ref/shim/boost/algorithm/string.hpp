/* Empty stand-in: the reference includes boost/algorithm/string.hpp in
 * Genome.cpp but calls nothing from it on the mapping path. */
#ifndef MSG_SHIM_ALGO_STRING_HPP
#define MSG_SHIM_ALGO_STRING_HPP
#include <string>
#endif
