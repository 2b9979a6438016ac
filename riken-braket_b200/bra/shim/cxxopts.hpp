// Project-written stand-in for the part of cxxopts that bra's main uses
// (bra/src/bra.cpp): Options with add_options()("s,long", description,
// value<T>()->default_value(...)), parse(argc, argv), count, operator[] ...
// as<T>() and help().  Options are given as --long value, --long=value or
// -s value.  Used to build the reference's code in this image, which does not
// have cxxopts.
#ifndef RBK_SHIM_CXXOPTS_HPP
#define RBK_SHIM_CXXOPTS_HPP

#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace cxxopts {

struct exception : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class value_base
{
 public:
  virtual ~value_base() = default;
  std::shared_ptr<value_base> default_value(std::string v)
  {
    default_ = std::move(v);
    has_default_ = true;
    return self_.lock();
  }
  bool has_default() const { return has_default_; }
  std::string const& default_text() const { return default_; }
  virtual bool is_boolean() const { return false; }
  std::weak_ptr<value_base> self_;

 private:
  std::string default_;
  bool has_default_ = false;
};

template <typename T>
class typed_value : public value_base { };

template <typename T>
inline std::shared_ptr<value_base> value()
{
  auto v = std::make_shared<typed_value<T>>();
  v->self_ = v;
  return v;
}

class option_value
{
 public:
  option_value() = default;
  explicit option_value(std::string text) : text_(std::move(text)), set_(true) { }
  template <typename T>
  T as() const
  {
    if (!set_) throw exception("option has no value");
    std::istringstream is(text_);
    T v{};
    if (!(is >> v)) throw exception("cannot parse option value '" + text_ + "'");
    return v;
  }

 private:
  std::string text_;
  bool set_ = false;
};
template <>
inline std::string option_value::as<std::string>() const
{
  if (!set_) throw exception("option has no value");
  return text_;
}
template <>
inline bool option_value::as<bool>() const { return set_ && text_ != "false"; }

class ParseResult
{
 public:
  std::size_t count(std::string const& name) const { return given_.count(name); }
  option_value const& operator[](std::string const& name) const
  {
    auto it = values_.find(name);
    if (it == values_.end()) throw exception("option '" + name + "' has no value");
    return it->second;
  }
  std::map<std::string, option_value> values_;
  std::map<std::string, int> given_;
};

class Options
{
  struct option {
    std::string shrt, lng, description;
    std::shared_ptr<value_base> value;
  };

 public:
  Options(std::string program, std::string description) : program_(std::move(program)), description_(std::move(description)) { }

  class adder
  {
   public:
    explicit adder(Options& o) : o_(o) { }
    adder& operator()(std::string const& names, std::string const& description,
                      std::shared_ptr<value_base> v = nullptr)
    {
      option opt;
      const auto comma = names.find(',');
      if (comma != std::string::npos) { opt.shrt = names.substr(0, comma); opt.lng = names.substr(comma + 1); }
      else opt.lng = names;
      opt.description = description;
      opt.value = v;
      o_.options_.push_back(opt);
      return *this;
    }

   private:
    Options& o_;
  };
  adder add_options() { return adder(*this); }

  ParseResult parse(int argc, char** argv) const
  {
    ParseResult r;
    for (const option& o : options_)
      if (o.value && o.value->has_default()) r.values_[o.lng] = option_value(o.value->default_text());
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i], name, text;
      bool has_text = false;
      if (a.rfind("--", 0) == 0) {
        name = a.substr(2);
        const auto eq = name.find('=');
        if (eq != std::string::npos) { text = name.substr(eq + 1); name = name.substr(0, eq); has_text = true; }
      } else if (a.size() > 1 && a[0] == '-') {
        name = a.substr(1);
      } else {
        throw exception("unexpected argument '" + a + "'");
      }
      const option* found = nullptr;
      for (const option& o : options_)
        if (o.lng == name || (!o.shrt.empty() && o.shrt == name)) found = &o;
      if (!found) throw exception("unknown option '" + a + "'");
      if (found->value && !has_text) {
        if (i + 1 >= argc) throw exception("option '" + a + "' needs a value");
        text = argv[++i];
      }
      r.values_[found->lng] = option_value(found->value ? text : std::string("true"));
      ++r.given_[found->lng];
    }
    return r;
  }

  std::string help() const
  {
    std::ostringstream os;
    os << description_ << "\nUsage:\n  " << program_ << " [OPTION...]\n\n";
    for (const option& o : options_) {
      os << "  " << (o.shrt.empty() ? "   " : "-" + o.shrt + ",") << " --" << o.lng;
      if (o.value) os << " arg";
      os << "    " << o.description;
      if (o.value && o.value->has_default()) os << " (default: " << o.value->default_text() << ")";
      os << '\n';
    }
    return os.str();
  }

 private:
  std::string program_, description_;
  std::vector<option> options_;
};

}  // namespace cxxopts

#endif
