// Stand-in for boost's concurrent_flat_map (boost is not in this image), for building
// the reference's Color_Table here (include/Color_Table.hpp:40-44 selects it unless
// USE_PARLAY_HASH is defined): a mutex-guarded hash map with the members Color_Table
// calls.  The map is live only in colored runs.  Test and baseline infrastructure only.
#pragma once

#include <cstddef>
#include <mutex>
#include <unordered_map>
#include <utility>

namespace boost {
namespace unordered {
template <typename K, typename V>
class concurrent_flat_map {
public:
    concurrent_flat_map() {}
    explicit concurrent_flat_map(std::size_t n) { m_.reserve(n); }
    std::size_t size() const { std::lock_guard<std::mutex> g(mu_); return m_.size(); }
    bool contains(const K& k) const { std::lock_guard<std::mutex> g(mu_); return m_.count(k) != 0; }
    // inserts (k, v) and returns true, or visits the present entry read-only and returns false
    template <typename F> bool emplace_or_cvisit(const K& k, const V& v, F f) {
        std::lock_guard<std::mutex> g(mu_);
        auto r = m_.emplace(k, v);
        if (!r.second) f(static_cast<const std::pair<const K, V>&>(*r.first));
        return r.second;
    }
    template <typename F> std::size_t visit(const K& k, F f) {
        std::lock_guard<std::mutex> g(mu_);
        auto it = m_.find(k);
        if (it == m_.end()) return 0;
        f(*it);
        return 1;
    }
    template <typename F> std::size_t cvisit(const K& k, F f) const {
        std::lock_guard<std::mutex> g(mu_);
        auto it = m_.find(k);
        if (it == m_.end()) return 0;
        f(static_cast<const std::pair<const K, V>&>(*it));
        return 1;
    }
    void clear() { std::lock_guard<std::mutex> g(mu_); m_.clear(); }

private:
    mutable std::mutex mu_;
    std::unordered_map<K, V> m_;
};
}  // namespace unordered
}  // namespace boost
