/* Minimal stand-in for boost::math::normal (pdf only), for the reference-oracle
 * build. Only the paired-end insert-size probability uses it; results there
 * are not pinned to Boost's last-ulp behaviour. */
#ifndef MSG_SHIM_NORMAL_HPP
#define MSG_SHIM_NORMAL_HPP
#include <cmath>
namespace boost { namespace math {
class normal {
public:
    normal(double m = 0, double s = 1) : m_(m), s_(s) {}
    double mean() const { return m_; }
    double standard_deviation() const { return s_; }
private:
    double m_, s_;
};
inline double pdf(const normal& d, double x) {
    const double z = (x - d.mean()) / d.standard_deviation();
    return std::exp(-0.5 * z * z) / (d.standard_deviation() * std::sqrt(2.0 * M_PI));
}
}}  // namespace boost::math
#endif
