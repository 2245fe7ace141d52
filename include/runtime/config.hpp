#pragma once
// String key/value configuration with typed getters.  Source-compatible
// with hytgraph::runtime::Config (reference include/runtime/config.hpp:9-24).

#include <cstdint>
#include <map>
#include <string>

namespace hytgraph::runtime {

class Config {
public:
    // Throws std::invalid_argument for an empty key.
    void set(std::string key, std::string value);
    [[nodiscard]] bool contains(const std::string &key) const;
    // Throws std::out_of_range("missing configuration key: <key>").
    [[nodiscard]] const std::string &get(const std::string &key) const;
    [[nodiscard]] std::string get_or(const std::string &key, std::string fallback) const;
    [[nodiscard]] std::int64_t get_int(const std::string &key) const;
    [[nodiscard]] double get_double(const std::string &key) const;
    // true/1/yes/on and false/0/no/off (case-insensitive); else invalid_argument.
    [[nodiscard]] bool get_bool(const std::string &key) const;
    [[nodiscard]] const std::map<std::string, std::string> &values() const noexcept { return values_; }

private:
    std::map<std::string, std::string> values_;
};

}  // namespace hytgraph::runtime
