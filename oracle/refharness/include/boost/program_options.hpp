// Test-harness stand-in for the parts of boost::program_options that the
// reference's src/user_options.h and src/user_options.cc name.  It is
// compile-only: the harness never parses a command line (it sets the
// User_options members directly, as a library caller of DTFE() does), so
// the parsing entry points (command_line_parser::run, parse_config_file)
// throw if they are ever reached.  The option tables that addOptions()
// declares are accepted and discarded.
#pragma once

#include <istream>
#include <map>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

class value_semantic {
 public:
  virtual ~value_semantic() {}
};

template <class T>
class typed_value : public value_semantic {
 public:
  explicit typed_value(T* store) : store_(store) {}
  typed_value* multitoken() { return this; }
  typed_value* zero_tokens() { return this; }
  typed_value* composing() { return this; }
  typed_value* default_value(const T&) { return this; }
  typed_value* default_value(const T&, const std::string&) { return this; }
  typed_value* implicit_value(const T&) { return this; }

 private:
  T* store_;
};

// boost returns a raw pointer that the options table then owns; the
// stand-in's tables keep them alive for the process (compile-only use)
template <class T>
typed_value<T>* value(T* store = nullptr) {
  static std::vector<std::unique_ptr<value_semantic>> keep;
  keep.emplace_back(new typed_value<T>(store));
  return static_cast<typed_value<T>*>(keep.back().get());
}

class options_description;

class options_description_easy_init {
 public:
  explicit options_description_easy_init(options_description* owner) : owner_(owner) {}
  options_description_easy_init& operator()(const char*, const char*) { return *this; }
  options_description_easy_init& operator()(const char*, const value_semantic*) { return *this; }
  options_description_easy_init& operator()(const char*, const value_semantic*, const char*) { return *this; }

 private:
  options_description* owner_;
};

class options_description {
 public:
  options_description() {}
  explicit options_description(const std::string& caption) : caption_(caption) {}
  options_description_easy_init add_options() { return options_description_easy_init(this); }
  options_description& add(const options_description&) { return *this; }
  friend std::ostream& operator<<(std::ostream& os, const options_description& d) { return os << d.caption_; }

 private:
  std::string caption_;
};

class positional_options_description {
 public:
  positional_options_description& add(const char*, int) { return *this; }
};

class variable_value {
 public:
  bool defaulted() const { return true; }
  bool empty() const { return true; }
  template <class T>
  const T& as() const {
    throw std::logic_error("program_options stand-in: no parsed values");
  }
};

class variables_map : public std::map<std::string, variable_value> {
 public:
  using std::map<std::string, variable_value>::operator[];
  const variable_value& operator[](const std::string& k) const {
    static const variable_value none;
    auto it = find(k);
    return it == end() ? none : it->second;
  }
};

struct parsed_options {};

class command_line_parser {
 public:
  command_line_parser(int, char**) {}
  command_line_parser& options(const options_description&) { return *this; }
  command_line_parser& positional(const positional_options_description&) { return *this; }
  command_line_parser& allow_unregistered() { return *this; }
  parsed_options run() { throw std::logic_error("program_options stand-in: command-line parsing is not built"); }
};

inline parsed_options parse_config_file(std::istream&, const options_description&, bool = false) {
  throw std::logic_error("program_options stand-in: config-file parsing is not built");
}

inline void store(const parsed_options&, variables_map&) {}
inline void notify(variables_map&) {}

}  // namespace program_options
}  // namespace boost
