#include "options.h"

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <vector>

namespace pbh {

static std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

// Cut a '#' comment that is not escaped and not inside single quotes.
static std::string strip_comment(const std::string& s) {
  bool q = false;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] == '\\') {
      ++i;
      continue;
    }
    if (s[i] == '\'') q = !q;
    if (s[i] == '#' && !q) return s.substr(0, i);
  }
  return s;
}

static std::string unescape(const std::string& v) {
  std::string t = trim(v);
  if (t.size() >= 2 && t.front() == '\'' && t.back() == '\'') return t.substr(1, t.size() - 2);
  std::string out;
  for (size_t i = 0; i < t.size(); ++i) {
    if (t[i] == '\\' && i + 1 < t.size()) {
      out.push_back(t[++i]);
      continue;
    }
    if (t[i] == ' ' || t[i] == '\t') break;  // an unescaped blank ends the value
    out.push_back(t[i]);
  }
  return out;
}

void OptionFile::load_stream(std::istream& in) {
  std::vector<std::string> stack;
  std::string line;
  while (std::getline(in, line)) {
    std::string s = trim(strip_comment(line));
    if (s.empty()) continue;
    if (s.front() == '[') {
      const size_t e = s.find(']');
      std::string sec = trim(s.substr(1, e == std::string::npos ? std::string::npos : e - 1));
      if (sec == "../") {
        if (!stack.empty()) stack.pop_back();
      } else if (sec.empty() || sec == "/") {
        stack.clear();
      } else {
        if (!sec.empty() && sec.back() == '/') sec.pop_back();
        if (sec.rfind("./", 0) == 0)
          stack.push_back(sec.substr(2));
        else {
          stack.clear();
          stack.push_back(sec);
        }
      }
      continue;
    }
    const size_t eq = s.find('=');
    if (eq == std::string::npos) continue;
    std::string key = trim(s.substr(0, eq));
    std::string prefix;
    for (const std::string& p : stack) prefix += p + "/";
    kv_[prefix + key] = unescape(s.substr(eq + 1));
  }
}

bool OptionFile::load_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) return false;
  load_stream(f);
  return true;
}

void OptionFile::load_text(const std::string& text) {
  std::istringstream in(text);
  load_stream(in);
}

std::string OptionFile::get(const std::string& key, const std::string& dflt) const {
  auto it = kv_.find(key);
  return it == kv_.end() ? dflt : it->second;
}

double OptionFile::get(const std::string& key, double dflt) const {
  auto it = kv_.find(key);
  if (it == kv_.end()) return dflt;
  char* end = nullptr;
  const double v = std::strtod(it->second.c_str(), &end);
  return end == it->second.c_str() ? dflt : v;
}

int OptionFile::get(const std::string& key, int dflt) const {
  auto it = kv_.find(key);
  if (it == kv_.end()) return dflt;
  char* end = nullptr;
  const long v = std::strtol(it->second.c_str(), &end, 10);
  return end == it->second.c_str() ? dflt : int(v);
}

}  // namespace pbh
