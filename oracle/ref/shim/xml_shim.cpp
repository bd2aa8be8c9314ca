// xml_shim.cpp -- ReaderXML / WriterXML of the reference Grains3D
// (src/Grains3D/Grains/XML3/include/ReaderXML.hh, WriterXML.hh) implemented
// over the minimal DOM of xercesc/dom/dom_shim.hpp, so that the reference
// sources compile without Xerces-C for the CPU oracle (test infrastructure).
// Lookup semantics follow the reference's XML3/src/ReaderXML.cpp: getNode on
// an element searches descendants, getNode on a node searches element
// children, getNodes(node) lists element children, node values are the text
// of the first child, getNodeNext is the second child node (text included).
#include "ReaderXML.hh"
#include "WriterXML.hh"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <vector>

namespace {

std::vector<DOMNode*> g_docs;  // parsed documents, alive until terminate()

struct Parser {
  const std::string& s;
  size_t i = 0;
  explicit Parser(const std::string& t) : s(t) {}
  bool starts(const char* p) const { return s.compare(i, std::strlen(p), p) == 0; }
  void skip_ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  void skip_until(const char* p) {
    size_t k = s.find(p, i);
    i = (k == std::string::npos) ? s.size() : k + std::strlen(p);
  }
  std::string name() {
    size_t b = i;
    while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/' && s[i] != '=') ++i;
    return s.substr(b, i - b);
  }
  static std::string unescape(const std::string& t) {
    std::string o;
    for (size_t k = 0; k < t.size(); ++k) {
      if (t[k] == '&') {
        size_t e = t.find(';', k);
        std::string ent = t.substr(k + 1, e - k - 1);
        if (ent == "lt") o += '<';
        else if (ent == "gt") o += '>';
        else if (ent == "amp") o += '&';
        else if (ent == "quot") o += '"';
        else if (ent == "apos") o += '\'';
        k = e;
      } else {
        o += t[k];
      }
    }
    return o;
  }
  // parses children of 'parent' until its closing tag (or end of input)
  void content(DOMNode* parent) {
    while (i < s.size()) {
      if (starts("<!--")) {
        skip_until("-->");
      } else if (starts("<?")) {
        skip_until("?>");
      } else if (starts("<!")) {
        skip_until(">");
      } else if (starts("</")) {
        skip_until(">");
        return;
      } else if (s[i] == '<') {
        ++i;
        DOMElement* e = new DOMElement();
        e->name = name();
        e->parent = parent;
        parent->children.push_back(e);
        for (;;) {
          skip_ws();
          if (i >= s.size()) return;
          if (starts("/>")) {
            i += 2;
            break;
          }
          if (s[i] == '>') {
            ++i;
            content(e);
            break;
          }
          std::string an = name();
          skip_ws();
          std::string av;
          if (i < s.size() && s[i] == '=') {
            ++i;
            skip_ws();
            char q = s[i++];
            size_t e2 = s.find(q, i);
            av = unescape(s.substr(i, e2 - i));
            i = e2 + 1;
          }
          e->attrs.push_back(std::make_pair(an, av));
        }
      } else {
        size_t e = s.find('<', i);
        if (e == std::string::npos) e = s.size();
        std::string txt = s.substr(i, e - i);
        i = e;
        // text nodes are kept, whitespace included, like a DOM parser does:
        // the reference reads the element after the first (whitespace) child
        // with getNodeNext (ConvexBuilderFactory::create)
        DOMNode* t = new DOMNode(DOMNode::TEXT_NODE);
        t->value = unescape(txt);
        t->parent = parent;
        parent->children.push_back(t);
      }
    }
  }
};

const std::string* attr(DOMNode* n, const std::string& name) {
  if (!n) return nullptr;
  for (auto& kv : n->attrs)
    if (kv.first == name) return &kv.second;
  return nullptr;
}

// ---- writer state ----
DOMElement* g_wroot = nullptr;

void write_node(std::ostream& o, DOMNode* n, int depth) {
  std::string ind(2 * depth, ' ');
  if (n->type == DOMNode::TEXT_NODE) {
    o << ind << n->value << "\n";
    return;
  }
  o << ind << "<" << n->name;
  for (auto& kv : n->attrs) o << " " << kv.first << "=\"" << kv.second << "\"";
  if (n->children.empty()) {
    o << "/>\n";
    return;
  }
  o << ">\n";
  for (DOMNode* c : n->children) write_node(o, c, depth + 1);
  o << ind << "</" << n->name << ">\n";
}
std::string num(double v) {
  std::ostringstream s;
  s.precision(17);
  s << v;
  return s.str();
}
}  // namespace

// ---------------------------------------------------------------------------
void ReaderXML::initialize() {}
void ReaderXML::terminate() {}

DOMNode* ReaderXML::getNode(DOMElement* root, string const& name) {
  if (!root) return nullptr;
  return root->descendants(name)->item(0);
}
DOMNode* ReaderXML::getNode(DOMNode* root, string const& name) {
  if (!root) return nullptr;
  DOMNodeList* l = root->child_list();
  for (XMLSize_t k = 0; k < l->getLength(); ++k)
    if (l->item(k)->name == name) return l->item(k);
  return nullptr;
}
double ReaderXML::getNodeAttr_Double(DOMNode* root, string const& name) {
  const std::string* v = attr(root, name);
  return v ? std::atof(v->c_str()) : 0.;
}
int ReaderXML::getNodeAttr_Int(DOMNode* root, string const& name) {
  const std::string* v = attr(root, name);
  return v ? std::atoi(v->c_str()) : 0;
}
string ReaderXML::getNodeAttr_String(DOMNode* root, string const& name) {
  const std::string* v = attr(root, name);
  return v ? *v : std::string();
}
bool ReaderXML::hasNodeAttr(DOMNode* root, string const& name) { return attr(root, name) != nullptr; }
string ReaderXML::getNodeName(DOMNode const* root) { return root ? root->name : std::string(); }
DOMNode* ReaderXML::getNodeNext(DOMNode* root) {
  if (!root || root->children.size() < 2) return nullptr;
  return root->children[1];
}
double ReaderXML::getNodeValue_Double(DOMNode* root) {
  if (!root || root->children.empty()) return 0.;
  return std::atof(root->children[0]->value.c_str());
}
string ReaderXML::getNodeValue_String(DOMNode* root) {
  if (!root || root->children.empty()) return "";
  return root->children[0]->value;
}
DOMNodeList* ReaderXML::getNodes(DOMElement* root, string const& name) {
  return root ? root->descendants(name) : nullptr;
}
DOMNodeList* ReaderXML::getNodes(DOMNode* root) { return root ? root->child_list() : nullptr; }
DOMElement* ReaderXML::getRoot(string const& xmlFile) {
  std::ifstream f(xmlFile.c_str());
  if (!f) {
    std::cerr << "XML file not found: " << xmlFile << std::endl;
    return nullptr;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string text = ss.str();
  DOMDocument* doc = new DOMDocument();
  Parser p(text);
  p.content(doc);
  g_docs.push_back(doc);
  for (DOMNode* c : doc->children)
    if (c->type == DOMNode::ELEMENT_NODE) return static_cast<DOMElement*>(c);
  return nullptr;
}

// ---------------------------------------------------------------------------
DOMElement* WriterXML::initialize(string const& root) {
  delete g_wroot;
  g_wroot = new DOMElement();
  g_wroot->name = root;
  return g_wroot;
}
void WriterXML::terminate(string const& file) {
  if (!g_wroot) return;
  std::ofstream o(file.c_str());
  o << "<?xml version=\"1.0\" encoding=\"iso-8859-1\"?>\n";
  write_node(o, g_wroot, 0);
  delete g_wroot;
  g_wroot = nullptr;
}
DOMElement* WriterXML::createNode(string const& name) {
  DOMElement* e = new DOMElement();
  e->name = name;
  if (g_wroot) {  // detached nodes are attached to the root so they are freed
    e->parent = g_wroot;
  }
  return e;
}
DOMElement* WriterXML::createNode(DOMElement* root, string const& name) {
  DOMElement* e = new DOMElement();
  e->name = name;
  e->parent = root;
  root->children.push_back(e);
  return e;
}
void WriterXML::createNodeAttr(DOMElement* root, string const& a, string const& v) {
  root->attrs.push_back(std::make_pair(a, v));
}
void WriterXML::createNodeAttr(DOMElement* root, string const& a, double v) {
  root->attrs.push_back(std::make_pair(a, num(v)));
}
void WriterXML::createNodeValue(DOMElement* root, string const& v) {
  DOMNode* t = new DOMNode(DOMNode::TEXT_NODE);
  t->value = v;
  t->parent = root;
  root->children.push_back(t);
}
void WriterXML::createNodeValue(DOMElement* root, double const& v) { createNodeValue(root, num(v)); }
