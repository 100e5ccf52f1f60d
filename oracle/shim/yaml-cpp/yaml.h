// Minimal stand-in for the part of yaml-cpp that NetFlux's ConfigParser uses.
//
// ORACLE-ONLY TEST INFRASTRUCTURE. yaml-cpp is not installed on this machine.
// This parses the input.yml subset NetFlux reads (ConfigParser.cpp:38-131):
//   key: scalar
//   key: [a, b, c]            (flow sequence of scalars)
//   key:
//     - name: value           (block sequence of single-key maps)
// with '#' comments and blank lines. It offers the yaml-cpp calls the parser
// makes: LoadFile, Node::operator[], explicit bool, as<T>, IsSequence, IsMap,
// size, Tag, iteration (sequence elements, or key/value pairs of a map) and
// the convert<T> customisation point.
#pragma once

#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace YAML {

class Node;
template <typename T>
struct convert;

class Node {
 public:
  enum class Kind { Undefined, Scalar, Sequence, Map };

 private:
  struct Data {
    Kind kind = Kind::Undefined;
    std::string scalar;
    std::vector<Node> seq;
    std::vector<std::pair<Node, Node>> map;
  };
  std::shared_ptr<Data> d_;

 public:
  Node() : d_(std::make_shared<Data>()) {}
  static Node scalar(const std::string& s) {
    Node n;
    n.d_->kind = Kind::Scalar;
    n.d_->scalar = s;
    return n;
  }
  static Node sequence() {
    Node n;
    n.d_->kind = Kind::Sequence;
    return n;
  }
  static Node mapping() {
    Node n;
    n.d_->kind = Kind::Map;
    return n;
  }
  void push_back(const Node& n) { d_->seq.push_back(n); }
  void insert(const std::string& k, const Node& v) { d_->map.emplace_back(scalar(k), v); }

  explicit operator bool() const { return d_->kind != Kind::Undefined; }
  bool IsDefined() const { return d_->kind != Kind::Undefined; }
  bool IsScalar() const { return d_->kind == Kind::Scalar; }
  bool IsSequence() const { return d_->kind == Kind::Sequence; }
  bool IsMap() const { return d_->kind == Kind::Map; }
  std::size_t size() const {
    return IsSequence() ? d_->seq.size() : (IsMap() ? d_->map.size() : 0);
  }
  std::string Tag() const { return "?"; }
  const std::string& Scalar() const { return d_->scalar; }

  Node operator[](const std::string& key) const {
    if (IsMap())
      for (const auto& kv : d_->map)
        if (kv.first.d_->scalar == key) return kv.second;
    return Node();
  }

  template <typename T>
  T as() const {
    if (!IsDefined()) throw std::runtime_error("yaml: conversion of an undefined node");
    if constexpr (std::is_same<T, std::string>::value) {
      if (!IsScalar()) throw std::runtime_error("yaml: bad conversion to string");
      return d_->scalar;
    } else if constexpr (std::is_same<T, bool>::value) {
      const std::string& s = d_->scalar;
      if (s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "on") return true;
      if (s == "false" || s == "False" || s == "FALSE" || s == "no" || s == "off") return false;
      throw std::runtime_error("yaml: bad conversion to bool: " + s);
    } else if constexpr (std::is_floating_point<T>::value) {
      if (!IsScalar()) throw std::runtime_error("yaml: bad conversion to number");
      std::size_t pos = 0;
      double v = std::stod(d_->scalar, &pos);
      if (pos != d_->scalar.size()) throw std::runtime_error("yaml: bad number: " + d_->scalar);
      return static_cast<T>(v);
    } else if constexpr (std::is_integral<T>::value) {
      if (!IsScalar()) throw std::runtime_error("yaml: bad conversion to integer");
      std::size_t pos = 0;
      long long v = std::stoll(d_->scalar, &pos);
      if (pos != d_->scalar.size()) throw std::runtime_error("yaml: bad integer: " + d_->scalar);
      return static_cast<T>(v);
    } else {
      T out;
      if (!convert<T>::decode(*this, out)) throw std::runtime_error("yaml: bad conversion");
      return out;
    }
  }

  class const_iterator;
  const_iterator begin() const;
  const_iterator end() const;
};

// Iteration yields values that are both a Node (sequence element) and a
// (key, value) pair (map entry), as yaml-cpp's iterator_value is.
struct iterator_value : public Node, public std::pair<Node, Node> {
  iterator_value(const Node& n, const std::pair<Node, Node>& kv) : Node(n), std::pair<Node, Node>(kv) {}
};

class Node::const_iterator {
  const Node* owner_;
  std::size_t i_;

 public:
  const_iterator(const Node* o, std::size_t i) : owner_(o), i_(i) {}
  iterator_value operator*() const {
    if (owner_->IsSequence()) return iterator_value(owner_->d_->seq[i_], std::pair<Node, Node>());
    return iterator_value(Node(), owner_->d_->map[i_]);
  }
  const_iterator& operator++() {
    ++i_;
    return *this;
  }
  bool operator!=(const const_iterator& o) const { return i_ != o.i_; }
  bool operator==(const const_iterator& o) const { return i_ == o.i_; }
};
inline Node::const_iterator Node::begin() const { return const_iterator(this, 0); }
inline Node::const_iterator Node::end() const { return const_iterator(this, size()); }

template <typename T>
struct convert;

namespace detail {
inline std::string trim(const std::string& s) {
  std::size_t a = s.find_first_not_of(" \t\r");
  if (a == std::string::npos) return "";
  std::size_t b = s.find_last_not_of(" \t\r");
  return s.substr(a, b - a + 1);
}
inline std::string strip_comment(const std::string& s) {
  bool q1 = false, q2 = false;
  for (std::size_t i = 0; i < s.size(); i++) {
    char c = s[i];
    if (c == '\'' && !q2) q1 = !q1;
    if (c == '"' && !q1) q2 = !q2;
    if (c == '#' && !q1 && !q2 && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
  }
  return s;
}
inline std::string unquote(const std::string& s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}
inline Node parse_value(const std::string& raw) {
  std::string v = trim(raw);
  if (v.size() >= 2 && v.front() == '[' && v.back() == ']') {
    Node seq = Node::sequence();
    std::string body = v.substr(1, v.size() - 2);
    std::stringstream ss(body);
    std::string item;
    while (std::getline(ss, item, ',')) {
      item = trim(item);
      if (!item.empty()) seq.push_back(Node::scalar(unquote(item)));
    }
    return seq;
  }
  return Node::scalar(unquote(v));
}
inline std::size_t indent_of(const std::string& s) {
  std::size_t n = 0;
  while (n < s.size() && s[n] == ' ') n++;
  return n;
}
}  // namespace detail

inline Node Load(std::istream& in) {
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(in, line)) {
    std::string s = detail::strip_comment(line);
    if (detail::trim(s).empty()) continue;
    lines.push_back(s);
  }
  Node root = Node::mapping();
  std::size_t i = 0;
  while (i < lines.size()) {
    const std::string& l = lines[i];
    if (detail::indent_of(l) != 0) throw std::runtime_error("yaml: unexpected indentation: " + l);
    std::size_t colon = l.find(':');
    if (colon == std::string::npos) throw std::runtime_error("yaml: expected 'key: value': " + l);
    std::string key = detail::trim(l.substr(0, colon));
    std::string rest = detail::trim(l.substr(colon + 1));
    i++;
    if (!rest.empty()) {
      root.insert(key, detail::parse_value(rest));
      continue;
    }
    // block: a sequence of "- item" lines (items may be "k: v" maps)
    Node seq = Node::sequence();
    while (i < lines.size() && detail::indent_of(lines[i]) > 0) {
      std::string item = detail::trim(lines[i]);
      if (item.empty() || item[0] != '-') throw std::runtime_error("yaml: expected '- item': " + lines[i]);
      item = detail::trim(item.substr(1));
      std::size_t c = item.find(':');
      if (c != std::string::npos && c + 1 <= item.size()) {
        Node m = Node::mapping();
        m.insert(detail::trim(item.substr(0, c)), detail::parse_value(item.substr(c + 1)));
        seq.push_back(m);
      } else {
        seq.push_back(Node::scalar(detail::unquote(item)));
      }
      i++;
    }
    root.insert(key, seq);
  }
  return root;
}

inline Node LoadFile(const std::string& filename) {
  std::ifstream in(filename);
  if (!in) throw std::runtime_error("bad file: " + filename);
  return Load(in);
}

}  // namespace YAML
