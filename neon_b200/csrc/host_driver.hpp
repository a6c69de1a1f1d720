// host_driver.hpp -- host-side pieces of neon's static_matrix that decide *what* the device does:
// boundary-value interpolation and adaptive load stepping.  Pure host C++, no CUDA.
#pragma once

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <queue>
#include <vector>

namespace nb2 {

// Boost.Math relative_difference(a, b) as neon's is_approx uses it
// (src/numeric/float_compare.hpp:20-32).
inline double relative_difference(double a, double b) {
    const double maxv = std::numeric_limits<double>::max();
    const double minv = std::numeric_limits<double>::min();
    if (std::isnan(a) || std::isnan(b)) return maxv;
    if (std::fabs(b) > maxv) return (std::fabs(a) > maxv && (a < 0) == (b < 0)) ? 0.0 : maxv;
    if (std::fabs(a) > maxv) return maxv;
    if (((a < 0) != (b < 0)) && a != 0 && b != 0) return maxv;
    a = std::fabs(a);
    b = std::fabs(b);
    if (a < minv) a = minv;
    if (b < minv) b = minv;
    return std::max(std::fabs((a - b) / a), std::fabs((a - b) / b));
}

inline bool is_approx(double x, double y, double abs_tol = 0.0, double rel_tol = 1e-10) {
    return relative_difference(x, y) <= rel_tol || std::fabs(x - y) <= abs_tol;
}

// mesh/boundary/boundary.cpp:36-85
struct TimeTable {
    std::vector<double> t, v;
    bool active(double time) const { return time >= t.front() && time <= t.back(); }
    double value(double time) const {
        for (size_t i = 0; i < t.size(); ++i)
            if (is_approx(t[i], time)) return v[i];
        for (size_t i = 0; i + 1 < t.size(); ++i)
            if (t[i] < time && time < t[i + 1]) {
                const double f = (time - t[i]) / (t[i + 1] - t[i]);
                return (1.0 - f) * v[i] + f * v[i + 1];
            }
        return v.back();
    }
};

// solver/adaptive_time_step.cpp:12-165.  update() returns false where the reference throws
// std::domain_error (cutback limit / increment below the minimum).
struct AdaptiveTimeStep {
    int increment_limit = 5;
    int successful_increments = 0, consecutive_converged = 0, consecutive_unconverged = 0;
    double initial_time = 1.0, final_time = 1.0, current_time = 1.0;
    double last_converged_time = 0.0, last_converged_time_step_size = 0.0;
    double minimum_increment = 0, maximum_increment = 0;
    bool is_applied = false;
    std::priority_queue<double, std::vector<double>, std::greater<double>> queue;

    void init(double period, double initial, double minimum, double maximum, bool adaptive,
              const std::vector<double>& history) {
        for (double t : history) queue.push(t);
        if (!queue.empty() && is_approx(queue.top(), 0.0)) queue.pop();
        initial_time = initial;
        minimum_increment = adaptive ? minimum : initial;
        maximum_increment = adaptive ? maximum : initial;
        final_time = period;
        current_time = std::min(queue.empty() ? initial : queue.top(), initial_time);
    }
    double step_time() const { return current_time; }
    double increment() const { return current_time - last_converged_time; }
    bool highly_nonlinear() const { return consecutive_unconverged > 0 || consecutive_converged < 4; }

    bool update(bool converged) {
        if (converged) {
            if (!queue.empty() && current_time >= queue.top()) queue.pop();
            last_converged_time_step_size = current_time - last_converged_time;
            last_converged_time = current_time;
            is_applied = is_approx(current_time, final_time) || queue.empty();
            consecutive_unconverged = 0;
            ++consecutive_converged;
            ++successful_increments;
            if (is_applied) return true;
            const double new_time = std::min(highly_nonlinear()
                                                 ? last_converged_time_step_size + current_time
                                                 : 2.0 * current_time,
                                             current_time + maximum_increment);
            current_time = std::min(queue.top(), std::min(new_time, final_time));
            return true;
        }
        const double dt = std::max(minimum_increment, (current_time - last_converged_time) * 0.5);
        current_time = last_converged_time + dt;
        if (current_time > final_time || current_time < 0.0) return false;
        ++consecutive_unconverged;
        consecutive_converged = 0;
        return consecutive_unconverged != increment_limit;
    }
};

}  // namespace nb2
