// Minimal stand-in for the part of Boost.Program_options that XPIR's server and client
// mains use: options_description with add_options()(name, [value,] help) chains and add(),
// value<T>([T* store])->default_value()->implicit_value(), parse_command_line ("--name v",
// "--name=v", "-n v", flags), store, notify, and variables_map count / operator[] / as<T>.
#ifndef XPIR_COMPAT_BOOST_PROGRAM_OPTIONS_HPP
#define XPIR_COMPAT_BOOST_PROGRAM_OPTIONS_HPP

#include <map>
#include <memory>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

class error : public std::logic_error {
 public:
  explicit error(const std::string &w) : std::logic_error(w) {}
};

// A parsed value: the text it came from, converted on demand.
class variable_value {
 public:
  variable_value() {}
  explicit variable_value(const std::string &text) : text_(text) {}
  template <class T>
  T as() const {
    T v;
    std::istringstream is(text_);
    is >> v;
    return v;
  }
  const std::string &text() const { return text_; }

 private:
  std::string text_;
};
template <>
inline std::string variable_value::as<std::string>() const {
  return text_;
}

class value_semantic {
 public:
  virtual ~value_semantic() {}
  virtual bool has_default() const = 0;
  virtual std::string default_text() const = 0;
  virtual bool has_implicit() const = 0;
  virtual std::string implicit_text() const = 0;
  virtual void store(const std::string &text) const = 0;  // into the bound variable, if any
};

template <class T>
class typed_value : public value_semantic {
 public:
  explicit typed_value(T *target) : target_(target) {}
  typed_value *default_value(const T &v) {
    default_ = text_of(v);
    has_default_ = true;
    return this;
  }
  typed_value *implicit_value(const T &v) {
    implicit_ = text_of(v);
    has_implicit_ = true;
    return this;
  }
  bool has_default() const override { return has_default_; }
  std::string default_text() const override { return default_; }
  bool has_implicit() const override { return has_implicit_; }
  std::string implicit_text() const override { return implicit_; }
  void store(const std::string &text) const override {
    if (target_) *target_ = variable_value(text).as<T>();
  }

 private:
  static std::string text_of(const T &v) {
    std::ostringstream os;
    os << v;
    return os.str();
  }
  T *target_;
  bool has_default_ = false, has_implicit_ = false;
  std::string default_, implicit_;
};

template <class T>
typed_value<T> *value() {
  return new typed_value<T>(nullptr);
}
template <class T>
typed_value<T> *value(T *target) {
  return new typed_value<T>(target);
}

struct option_description {
  std::string long_name, short_name, help;
  std::shared_ptr<value_semantic> semantic;  // null for a flag
};

class options_description {
 public:
  options_description() {}
  explicit options_description(const std::string &caption) : caption_(caption) {}

  class easy_init {
   public:
    explicit easy_init(options_description *o) : o_(o) {}
    easy_init &operator()(const char *name, const char *help) {
      o_->add_one(name, nullptr, help);
      return *this;
    }
    easy_init &operator()(const char *name, value_semantic *s, const char *help) {
      o_->add_one(name, s, help);
      return *this;
    }

   private:
    options_description *o_;
  };
  easy_init add_options() { return easy_init(this); }
  options_description &add(const options_description &other) {
    for (const auto &d : other.options_) options_.push_back(d);
    return *this;
  }
  const std::vector<option_description> &options() const { return options_; }
  const std::string &caption() const { return caption_; }

  // The option of a "--long" or "-short" name, or null.  As with Boost's default style, a
  // long name may be abbreviated to any unambiguous prefix ("--alpha" for "--alphaMax").
  const option_description *find(const std::string &name, bool is_long) const {
    for (const auto &d : options_)
      if ((is_long ? d.long_name : d.short_name) == name) return &d;
    for (const auto &d : options_)
      if (d.short_name == name || d.long_name == name) return &d;
    if (!is_long) return nullptr;
    const option_description *hit = nullptr;
    for (const auto &d : options_)
      if (d.long_name.compare(0, name.size(), name) == 0) {
        if (hit) return nullptr;  // ambiguous
        hit = &d;
      }
    return hit;
  }

 private:
  void add_one(const char *name, value_semantic *s, const char *help) {
    option_description d;
    std::string n(name);
    const size_t comma = n.find(',');
    d.long_name = n.substr(0, comma);
    if (comma != std::string::npos) d.short_name = n.substr(comma + 1);
    d.help = help ? help : "";
    d.semantic.reset(s);
    options_.push_back(d);
  }
  std::string caption_;
  std::vector<option_description> options_;
};

inline std::ostream &operator<<(std::ostream &os, const options_description &od) {
  if (!od.caption().empty()) os << od.caption() << ":\n";
  for (const auto &d : od.options()) {
    os << "  --" << d.long_name;
    if (!d.short_name.empty()) os << " [ -" << d.short_name << " ]";
    if (d.semantic) os << " arg";
    if (d.semantic && d.semantic->has_default()) os << " (=" << d.semantic->default_text() << ")";
    os << "\t" << d.help << "\n";
  }
  return os;
}

class variables_map : public std::map<std::string, variable_value> {
 public:
  // Values bound to variables, applied by notify().
  std::vector<std::pair<std::shared_ptr<value_semantic>, std::string>> pending;
};

struct parsed_options {
  std::vector<std::pair<const option_description *, std::string>> given;  // text "" for flags
  const options_description *desc = nullptr;
};

inline parsed_options parse_command_line(int argc, char *argv[], const options_description &od) {
  parsed_options p;
  p.desc = &od;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') throw error("unexpected positional argument " + a);
    const bool is_long = a[1] == '-';
    std::string name = a.substr(is_long ? 2 : 1), text;
    bool has_text = false;
    const size_t eq = name.find('=');
    if (eq != std::string::npos) {
      text = name.substr(eq + 1);
      name = name.substr(0, eq);
      has_text = true;
    }
    const option_description *d = od.find(name, is_long);
    if (!d) throw error("unrecognised option " + a);
    if (d->semantic && !has_text) {
      if (i + 1 < argc && argv[i + 1][0] != '-') {
        text = argv[++i];
      } else if (d->semantic->has_implicit()) {
        text = d->semantic->implicit_text();
      } else {
        throw error("option " + a + " needs a value");
      }
    }
    p.given.push_back(std::make_pair(d, text));
  }
  return p;
}

inline void store(const parsed_options &p, variables_map &vm) {
  for (const auto &g : p.given) {
    vm[g.first->long_name] = variable_value(g.second);
    if (g.first->semantic) vm.pending.push_back(std::make_pair(g.first->semantic, g.second));
  }
  // Defaults of the options not given.
  for (const auto &d : p.desc->options())
    if (d.semantic && d.semantic->has_default() && !vm.count(d.long_name)) {
      vm[d.long_name] = variable_value(d.semantic->default_text());
      vm.pending.push_back(std::make_pair(d.semantic, d.semantic->default_text()));
    }
}

inline void notify(variables_map &vm) {
  for (const auto &p : vm.pending) p.first->store(p.second);
}

}  // namespace program_options
}  // namespace boost

#endif
