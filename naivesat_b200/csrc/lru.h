// lru.h -- a bounded map that forgets its least recently used entries.
#pragma once
#include <cstddef>
#include <iterator>
#include <list>
#include <map>
#include <utility>
#include <vector>

namespace nsat {

// Holds at most `capacity` entries.  find() and put() make an entry the most
// recently used; put() evicts from the other end and hands the evicted values
// to the caller, who decides where they are destroyed (for example outside a
// lock, or with a particular device current).
template <typename K, typename V>
class LruMap {
public:
    explicit LruMap(size_t capacity = 1) : cap_(capacity ? capacity : 1) {}

    size_t capacity() const { return cap_; }
    size_t size() const { return items_.size(); }

    // The value stored for k, or nullptr.
    V* find(const K& k) {
        auto it = index_.find(k);
        if (it == index_.end()) return nullptr;
        items_.splice(items_.begin(), items_, it->second);
        return &it->second->second;
    }

    // Stores v for k (replacing an existing value, which is evicted too).
    void put(const K& k, V v, std::vector<V>* evicted) {
        auto it = index_.find(k);
        if (it != index_.end()) {
            std::swap(it->second->second, v);
            if (evicted) evicted->push_back(std::move(v));
            items_.splice(items_.begin(), items_, it->second);
            return;
        }
        items_.emplace_front(k, std::move(v));
        index_[k] = items_.begin();
        trim(evicted);
    }

    void set_capacity(size_t capacity, std::vector<V>* evicted) {
        cap_ = capacity ? capacity : 1;
        trim(evicted);
    }

private:
    void trim(std::vector<V>* evicted) {
        while (items_.size() > cap_) {
            auto last = std::prev(items_.end());
            if (evicted) evicted->push_back(std::move(last->second));
            index_.erase(last->first);
            items_.pop_back();
        }
    }

    size_t cap_;
    std::list<std::pair<K, V>> items_;   // most recently used first
    std::map<K, typename std::list<std::pair<K, V>>::iterator> index_;
};

}  // namespace nsat
