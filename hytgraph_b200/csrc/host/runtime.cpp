// Runtime support: Config, log, Result JSON (reference src/runtime/*.cpp).
#include "runtime/config.hpp"
#include "runtime/logging.hpp"
#include "runtime/result.hpp"

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <stdexcept>

namespace hytgraph::runtime {

// --------------------------------- Config --------------------------------

void Config::set(std::string key, std::string value) {
    if (key.empty()) throw std::invalid_argument("configuration key must not be empty");
    values_[std::move(key)] = std::move(value);
}

bool Config::contains(const std::string &key) const { return values_.count(key) != 0; }

const std::string &Config::get(const std::string &key) const {
    const auto it = values_.find(key);
    if (it == values_.end()) throw std::out_of_range("missing configuration key: " + key);
    return it->second;
}

std::string Config::get_or(const std::string &key, std::string fallback) const {
    const auto it = values_.find(key);
    return it == values_.end() ? fallback : it->second;
}

std::int64_t Config::get_int(const std::string &key) const { return std::stoll(get(key)); }
double Config::get_double(const std::string &key) const { return std::stod(get(key)); }

bool Config::get_bool(const std::string &key) const {
    std::string v = get(key);
    std::transform(v.begin(), v.end(), v.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    if (v == "true" || v == "1" || v == "yes" || v == "on") return true;
    if (v == "false" || v == "0" || v == "no" || v == "off") return false;
    throw std::invalid_argument("invalid boolean configuration value for key: " + key);
}

// --------------------------------- log -----------------------------------

namespace {
std::mutex g_log_mutex;
LogLevel g_log_level = LogLevel::Info;

const char *level_name(LogLevel l) {
    switch (l) {
        case LogLevel::Debug: return "DEBUG";
        case LogLevel::Info: return "INFO";
        case LogLevel::Warning: return "WARN";
        case LogLevel::Error: return "ERROR";
    }
    return "UNKNOWN";
}
}  // namespace

void set_log_level(LogLevel level) noexcept {
    std::lock_guard<std::mutex> lock(g_log_mutex);
    g_log_level = level;
}

void log(LogLevel level, std::string_view message) {
    std::lock_guard<std::mutex> lock(g_log_mutex);
    if (static_cast<int>(level) < static_cast<int>(g_log_level)) return;
    const std::time_t t = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
    std::tm utc{};
    gmtime_r(&t, &utc);
    std::cerr << '[' << std::put_time(&utc, "%Y-%m-%dT%H:%M:%SZ") << "] " << level_name(level) << ' ' << message
              << '\n';
}

// --------------------------------- Result --------------------------------

namespace {
std::string escape(const std::string &s) {
    std::string o;
    o.reserve(s.size());
    for (const char c : s) {
        switch (c) {
            case '"': o += "\\\""; break;
            case '\\': o += "\\\\"; break;
            case '\n': o += "\\n"; break;
            case '\r': o += "\\r"; break;
            case '\t': o += "\\t"; break;
            default: o += c;
        }
    }
    return o;
}
}  // namespace

std::string result_to_json(const Result &r) {
    std::ostringstream o;
    o << std::setprecision(17);
    o << "{\n  \"schema_version\": \"" << escape(r.schema_version) << "\",\n  \"experiment_id\": \""
      << escape(r.experiment_id) << "\",\n  \"status\": \"" << escape(r.status) << "\",\n  \"timestamp_utc\": \""
      << escape(r.timestamp_utc) << "\",\n  \"git_commit\": \"" << escape(r.git_commit) << "\",\n  \"config\": {";
    bool first = true;
    for (const auto &[k, v] : r.config) {
        o << (first ? "" : ",") << "\n    \"" << escape(k) << "\": \"" << escape(v) << '"';
        first = false;
    }
    o << (r.config.empty() ? "" : "\n") << "  },\n  \"measurements\": {";
    first = true;
    for (const auto &[k, v] : r.measurements) {
        o << (first ? "" : ",") << "\n    \"" << escape(k) << "\": ";
        if (std::isfinite(v))
            o << v;
        else
            o << "null";  // JSON has no inf/nan
        first = false;
    }
    o << (r.measurements.empty() ? "" : "\n") << "  }\n}\n";
    return o.str();
}

bool write_result_json(const Result &r, const std::string &path) {
    std::ofstream f(path);
    if (!f) return false;
    f << result_to_json(r);
    return static_cast<bool>(f);
}

}  // namespace hytgraph::runtime
