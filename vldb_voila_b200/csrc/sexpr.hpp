/*
 * S-expression reader for plan text.
 *
 * Plan text is the serialised form of a relational plan (the reference's relalg tree,
 * relalg.hpp:12-178) that crosses the C ABI:
 *
 *   expr := (const INT) | (col NAME) | (fun NAME expr*) | (assign NAME expr)
 *   op   := (scan TABLE (COLUMN*))
 *         | (select expr op)
 *         | (project (expr*) op)
 *         | (aggr hash|global (key-expr*) (aggregate-expr*) op)
 *         | (join join01|joinN (probe-key*) (probe-payload*) probe-op
 *                              (build-key*) (build-payload*) build-op)
 *
 * Aggregates are (fun sum expr) and (fun count).  Atoms are separated by white space and
 * parentheses; there is no quoting.
 */
#ifndef VOILA_B200_SEXPR_HPP
#define VOILA_B200_SEXPR_HPP

#include <cctype>
#include <stdexcept>
#include <string>
#include <vector>

namespace vc_sexpr {

struct Node {
	bool atom = false;
	std::string text;
	std::vector<Node> kids;

	const std::string& head() const {
		if (atom || kids.empty() || !kids[0].atom) {
			throw std::invalid_argument("plan: expected (name ...) list");
		}
		return kids[0].text;
	}
	const Node& at(size_t i) const {
		if (atom || i >= kids.size()) {
			throw std::invalid_argument("plan: missing element " + std::to_string(i) +
				(atom ? " in atom '" + text + "'" : " in list '" + (kids.empty() ? std::string("()") : kids[0].text) + "'"));
		}
		return kids[i];
	}
	const std::string& atom_text(size_t i) const {
		const Node& n = at(i);
		if (!n.atom) {
			throw std::invalid_argument("plan: expected an atom at position " + std::to_string(i));
		}
		return n.text;
	}
};

class Reader {
	const std::string& s;
	size_t pos = 0;

	void skip() {
		while (pos < s.size() && std::isspace((unsigned char)s[pos])) {
			pos++;
		}
	}

public:
	explicit Reader(const std::string& src) : s(src) {}

	Node read() {
		skip();
		if (pos >= s.size()) {
			throw std::invalid_argument("plan: unexpected end of text");
		}
		Node n;
		if (s[pos] == '(') {
			pos++;
			for (;;) {
				skip();
				if (pos >= s.size()) {
					throw std::invalid_argument("plan: missing ')'");
				}
				if (s[pos] == ')') {
					pos++;
					break;
				}
				n.kids.push_back(read());
			}
			return n;
		}
		if (s[pos] == ')') {
			throw std::invalid_argument("plan: unexpected ')'");
		}
		n.atom = true;
		size_t start = pos;
		while (pos < s.size() && !std::isspace((unsigned char)s[pos]) && s[pos] != '(' && s[pos] != ')') {
			pos++;
		}
		n.text = s.substr(start, pos - start);
		return n;
	}

	bool at_end() {
		skip();
		return pos >= s.size();
	}
};

inline Node parse(const std::string& text)
{
	Reader r(text);
	Node n = r.read();
	if (!r.at_end()) {
		throw std::invalid_argument("plan: trailing text after the plan");
	}
	return n;
}

} // namespace vc_sexpr

#endif
