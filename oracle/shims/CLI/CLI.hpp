// Interface shim for the subset of CLI11 the reference tools use
// (App::add_option / add_flag / Option::group / Option::required / App::parse /
// App::exit / ParseError), written for this project because CLI11 is not
// available offline.  Options take their value from the next argument or from
// "--name=value"; flags bound to a bool are set to true, flags bound to any
// other type take an "=value" suffix when one is given.
#pragma once
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace CLI {

class ParseError : public std::runtime_error {
 public:
  ParseError(const std::string &msg, int code)
      : std::runtime_error(msg), code_(code) {}
  int get_exit_code() const { return code_; }

 private:
  int code_;
};

class Option {
 public:
  Option(std::vector<std::string> names, std::function<void(const std::string &)> set,
         bool flag, bool bool_flag)
      : names_(std::move(names)), set_(std::move(set)), flag_(flag), bool_flag_(bool_flag) {}
  Option *group(const std::string &) { return this; }
  Option *required(bool r = true) {
    required_ = r;
    return this;
  }
  Option *check(...) { return this; }

  std::vector<std::string> names_;
  std::function<void(const std::string &)> set_;
  bool flag_, bool_flag_;
  bool required_ = false;
  bool seen_ = false;
};

namespace detail {
inline std::vector<std::string> split_names(const std::string &spec) {
  std::vector<std::string> out;
  std::stringstream ss(spec);
  std::string tok;
  while (std::getline(ss, tok, ',')) {
    while (!tok.empty() && tok.front() == ' ') tok.erase(tok.begin());
    if (!tok.empty()) out.push_back(tok);
  }
  return out;
}

template <typename T>
void assign(T &var, const std::string &text) {
  if constexpr (std::is_same_v<T, std::string>) {
    var = text;
  } else if constexpr (std::is_same_v<T, bool>) {
    var = !(text == "0" || text == "false" || text == "off");
  } else {
    std::istringstream is(text);
    T tmp{};
    is >> tmp;
    if (is.fail()) throw ParseError("invalid value: " + text, 106);
    var = tmp;
  }
}
}  // namespace detail

class App {
 public:
  App() = default;
  explicit App(const std::string &) {}

  template <typename T>
  Option *add_option(const std::string &spec, T &var, const std::string & = "") {
    opts_.push_back(std::make_unique<Option>(
        detail::split_names(spec),
        [&var](const std::string &t) { detail::assign(var, t); }, false, false));
    return opts_.back().get();
  }

  template <typename T>
  Option *add_flag(const std::string &spec, T &var, const std::string & = "") {
    constexpr bool is_bool = std::is_same_v<T, bool>;
    opts_.push_back(std::make_unique<Option>(
        detail::split_names(spec),
        [&var](const std::string &t) { detail::assign(var, t); }, true, is_bool));
    return opts_.back().get();
  }

  void parse(int argc, char **argv) {
    for (int i = 1; i < argc; ++i) {
      std::string arg = argv[i];
      if (arg == "-h" || arg == "--help") throw ParseError("help", 0);
      std::string name = arg, value;
      bool has_value = false;
      auto eq = arg.find('=');
      if (arg.rfind("--", 0) == 0 && eq != std::string::npos) {
        name = arg.substr(0, eq);
        value = arg.substr(eq + 1);
        has_value = true;
      }
      Option *o = find(name);
      if (!o) throw ParseError("unknown argument: " + arg, 109);
      o->seen_ = true;
      if (o->flag_) {
        o->set_(has_value ? value : (o->bool_flag_ ? "true" : ""));
        continue;
      }
      if (!has_value) {
        if (i + 1 >= argc) throw ParseError("missing value for " + name, 106);
        value = argv[++i];
      }
      o->set_(value);
    }
    for (auto &o : opts_)
      if (o->required_ && !o->seen_)
        throw ParseError("required option missing: " + o->names_.front(), 106);
  }

  int exit(const ParseError &e) const {
    if (e.get_exit_code() != 0) std::cerr << e.what() << std::endl;
    return e.get_exit_code();
  }

 private:
  Option *find(const std::string &name) {
    for (auto &o : opts_)
      for (auto &n : o->names_)
        if (n == name) return o.get();
    return nullptr;
  }
  std::vector<std::unique_ptr<Option>> opts_;
};

}  // namespace CLI
