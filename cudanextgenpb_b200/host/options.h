// options.prm reader: the subset of GetPot syntax the reference's option files
// use (data/options.prm, test/options.prm): "[section]" ... "[../]" blocks,
// "key = value" pairs, '#' comments, values with backslash-escaped blanks
// ("-p\ ssor\ -tol\ 1.e-6") or quoted with single quotes.  Keys are stored as
// "section/key", the form parse_options queries (src/pb_class.cpp:809-978).
#pragma once
#include <istream>
#include <map>
#include <string>

namespace pbh {

class OptionFile {
 public:
  bool load_file(const std::string& path);
  void load_text(const std::string& text);
  void load_stream(std::istream& in);
  bool has(const std::string& key) const { return kv_.count(key) != 0; }
  std::string get(const std::string& key, const std::string& dflt) const;
  double get(const std::string& key, double dflt) const;
  int get(const std::string& key, int dflt) const;
  void set(const std::string& key, const std::string& value) { kv_[key] = value; }
  const std::map<std::string, std::string>& all() const { return kv_; }

 private:
  std::map<std::string, std::string> kv_;
};

}  // namespace pbh
