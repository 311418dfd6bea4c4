// Reference-surface shim: the case configuration (src/core/config.hpp):
// "key = value" lines, '#' and ';' start comments, overrides by set();
// getters record the keys they read so that unused() can report the rest.
#pragma once

#include <map>
#include <set>
#include <string>
#include <vector>

#include "core/precision.hpp"

namespace wfe {

class Config {
 public:
  bool load(const std::string& path);
  void set(const std::string& key, const std::string& val) { kv_[key] = val; }
  bool has(const std::string& key) const { return kv_.count(key) > 0; }
  real get_real(const std::string& key, real def) const;
  int get_int(const std::string& key, int def) const;
  std::string get_str(const std::string& key, const std::string& def) const;
  const std::map<std::string, std::string>& raw() const { return kv_; }
  // keys no getter has read (the projection keys of the prep tool excepted)
  std::vector<std::string> unused() const;
  // the configuration as "key = value" lines (what wfe_case_create_text reads)
  std::string text() const;

 private:
  std::map<std::string, std::string> kv_;
  mutable std::set<std::string> used_;
};

}  // namespace wfe
