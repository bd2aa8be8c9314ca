// dom_shim.hpp -- a minimal DOM (elements, attributes, text) standing in for
// Xerces-C when the reference Grains3D sources are compiled as the CPU
// oracle (test infrastructure).  Only what the reference's ReaderXML /
// WriterXML interface and its callers use is provided.
#ifndef GRAINS_ORACLE_DOM_SHIM_HPP
#define GRAINS_ORACLE_DOM_SHIM_HPP
#include <cstddef>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace xercesc {
typedef std::size_t XMLSize_t;
typedef char16_t XMLCh;

class DOMNodeList;

class DOMNode {
 public:
  enum NodeType { ELEMENT_NODE = 1, TEXT_NODE = 3, DOCUMENT_NODE = 9 };
  explicit DOMNode(NodeType t) : type(t) {}
  virtual ~DOMNode();
  NodeType getNodeType() const { return type; }
  NodeType type;
  std::string name;                          // element tag
  std::string value;                         // text content
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<DOMNode*> children;            // owned
  DOMNode* parent = nullptr;
  DOMNodeList* child_list();                 // element children (cached)
  DOMNodeList* descendants(const std::string& tag);  // cached per tag
 private:
  std::unique_ptr<DOMNodeList> children_cache_;
  std::map<std::string, std::unique_ptr<DOMNodeList>> desc_cache_;
};

class DOMElement : public DOMNode {
 public:
  DOMElement() : DOMNode(ELEMENT_NODE) {}
};

class DOMDocument : public DOMNode {
 public:
  DOMDocument() : DOMNode(DOCUMENT_NODE) {}
};

class DOMNodeList {
 public:
  std::vector<DOMNode*> nodes;
  XMLSize_t getLength() const { return nodes.size(); }
  DOMNode* item(XMLSize_t i) const { return i < nodes.size() ? nodes[i] : nullptr; }
};

inline DOMNode::~DOMNode() {
  for (DOMNode* c : children) delete c;
}
inline DOMNodeList* DOMNode::child_list() {
  if (!children_cache_) {
    children_cache_.reset(new DOMNodeList());
    for (DOMNode* c : children)
      if (c->type == ELEMENT_NODE) children_cache_->nodes.push_back(c);
  }
  return children_cache_.get();
}
inline void dom_shim_collect(DOMNode* n, const std::string& tag, std::vector<DOMNode*>& out) {
  for (DOMNode* c : n->children)
    if (c->type == DOMNode::ELEMENT_NODE) {
      if (c->name == tag) out.push_back(c);
      dom_shim_collect(c, tag, out);
    }
}
inline DOMNodeList* DOMNode::descendants(const std::string& tag) {
  auto it = desc_cache_.find(tag);
  if (it != desc_cache_.end()) return it->second.get();
  DOMNodeList* l = new DOMNodeList();
  dom_shim_collect(this, tag, l->nodes);
  desc_cache_[tag].reset(l);
  return l;
}
}  // namespace xercesc

#define XERCES_CPP_NAMESPACE_USE using namespace xercesc;
#define XERCES_STD_QUALIFIER std::
#endif
