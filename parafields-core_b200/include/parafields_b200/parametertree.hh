// parametertree.hh -- the subset of Dune::ParameterTree that parafields-core's
// configuration code uses (get<T>(key), get<T>(key, default), operator[], INI files),
// so configurations written for the reference (test/fieldtest.cc:12-17,
// randomfield.hh:78-84) drive the B200 path unchanged.
#pragma once

#include <array>
#include <cctype>
#include <fstream>
#include <map>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace parafields_b200 {

class ParameterTree {
  std::map<std::string, std::string> values_;

  static std::string trim(const std::string& s) {
    const auto a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const auto b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
  }

  template <typename T>
  static T parse_one(const std::string& key, const std::string& text) {
    std::istringstream in(text);
    T v{};
    in >> v;
    if (in.fail()) throw std::runtime_error{"cannot parse value \"" + text + "\" of key " + key};
    return v;
  }

 public:
  std::string& operator[](const std::string& key) { return values_[key]; }
  bool hasKey(const std::string& key) const { return values_.count(key) != 0; }

  // INI text: "key = value" lines, "[section]" prefixes following keys with "section."
  void parseIni(const std::string& text) {
    std::istringstream in(text);
    std::string line, prefix;
    while (std::getline(in, line)) {
      const auto hash = line.find_first_of("#;");
      if (hash != std::string::npos) line = line.substr(0, hash);
      line = trim(line);
      if (line.empty()) continue;
      if (line.front() == '[' && line.back() == ']') {
        prefix = trim(line.substr(1, line.size() - 2));
        if (!prefix.empty()) prefix += ".";
        continue;
      }
      const auto eq = line.find('=');
      if (eq == std::string::npos) throw std::runtime_error{"malformed configuration line: " + line};
      std::string val = trim(line.substr(eq + 1));
      if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
      values_[prefix + trim(line.substr(0, eq))] = val;
    }
  }

  // Dune::ParameterTree::report layout: keys without a section as key = "value", then one
  // "[ section ]" block per section (sorted) with its keys relative to it
  void report(std::ostream& out) const {
    std::map<std::string, std::map<std::string, std::string>> sections;
    for (const auto& kv : values_) {
      const auto dot = kv.first.rfind('.');
      if (dot == std::string::npos)
        sections[""][kv.first] = kv.second;
      else
        sections[kv.first.substr(0, dot)][kv.first.substr(dot + 1)] = kv.second;
    }
    for (const auto& sec : sections) {
      if (!sec.first.empty()) out << "[ " << sec.first << " ]\n";
      for (const auto& kv : sec.second) out << kv.first << " = \"" << kv.second << "\"\n";
    }
  }

  void readIniFile(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error{"cannot open configuration file " + path};
    std::stringstream ss;
    ss << f.rdbuf();
    parseIni(ss.str());
  }

  std::string raw(const std::string& key) const {
    auto it = values_.find(key);
    if (it == values_.end()) throw std::runtime_error{"missing configuration key " + key};
    return it->second;
  }

  template <typename T>
  T get(const std::string& key) const {
    return convert<T>(key, raw(key));
  }

  template <typename T>
  T get(const std::string& key, const T& def) const {
    auto it = values_.find(key);
    return it == values_.end() ? def : convert<T>(key, it->second);
  }

  std::string get(const std::string& key, const char* def) const { return get<std::string>(key, std::string(def)); }

  std::vector<double> getVector(const std::string& key) const {
    std::istringstream in(raw(key));
    std::vector<double> v;
    double x;
    while (in >> x) v.push_back(x);
    return v;
  }

 private:
  template <typename T>
  struct tag {};

  template <typename T>
  static T convert(const std::string& key, const std::string& text) {
    return convert_impl(key, text, tag<T>{});
  }
  static std::string convert_impl(const std::string&, const std::string& text, tag<std::string>) { return text; }
  static bool convert_impl(const std::string& key, const std::string& text, tag<bool>) {
    std::string t;
    for (char c : text) t += (char)std::tolower((unsigned char)c);
    if (t == "true" || t == "yes" || t == "1") return true;
    if (t == "false" || t == "no" || t == "0") return false;
    throw std::runtime_error{"cannot parse boolean \"" + text + "\" of key " + key};
  }
  template <typename T>
  static T convert_impl(const std::string& key, const std::string& text, tag<T>) {
    return parse_one<T>(key, text);
  }
  template <typename T, std::size_t N>
  static std::array<T, N> convert_impl(const std::string& key, const std::string& text, tag<std::array<T, N>>) {
    std::istringstream in(text);
    std::array<T, N> a{};
    for (std::size_t i = 0; i < N; i++) {
      in >> a[i];
      if (in.fail()) throw std::runtime_error{"key " + key + " needs " + std::to_string(N) + " values"};
    }
    return a;
  }
};

}  // namespace parafields_b200
