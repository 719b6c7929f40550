// Device-resident pipeline runner: a pipeline document (the reference's
// *.cpipe.json, schema v0.4) planned once and run frame after frame on the
// host's CUDA stream over planner slots kept on the device.
//
// Load follows the reference Pipeline::load (src/cpipe/runtime/Pipeline.cpp:368-601):
//   * version "0.4", nodes / edges / inputs present (else CPIPE_FAILED);
//   * "com.cpipe.precision_convert" is reserved for implicit nodes
//     (CPIPE_BAD_INDEX); node types resolve in this library's registry
//     (unknown: CPIPE_BAD_INDEX); params checked against the manifest
//     (unknown name, wrong type, outside range or enum: CPIPE_BAD_INDEX,
//     Pipeline.cpp:214-300);
//   * edges "node.port"; a dangling endpoint is CPIPE_BAD_INDEX;
//   * topological order by Kahn's algorithm over the document order, a cycle
//     is CPIPE_FAILED;
//   * every step an input port requires must be set upstream, and colour
//     roles must agree on every edge (CPIPE_NEED_METADATA, Pipeline.cpp:469-504);
//   * precision planning as PrecisionPlanner::auto_insert: an edge whose
//     precisions do not intersect gets an implicit precision_convert when the
//     direct conversion exists (R16_UINT->R32_SFLOAT, R32_SFLOAT->RGBA16F,
//     RGBA16F->RGBA8 / RGBA16 unorm), else CPIPE_BAD_PRECISION;
//   * output formats as output_layout_for_node (Pipeline.cpp:127-172).
// An optional `until` node id restricts the plan to that node and what it
// depends on, so a document that ends in nodes outside this library (the HEIF
// writers) can run its device prefix.
//
// Run differs from Pipeline::run_bound (Pipeline.cpp:629-792) in where the
// buffers live and when the host waits: instead of a fresh CpuBuffer per node
// and a synchronous node-by-node walk, each node's output is a view over a
// device slot of the memory plan (MemoryPlanner::plan_graph,
// MemoryPlanner.cpp:188-219: live ranges over the topological order, slots
// shared by buffers whose ranges do not meet, first fit in order), the slots
// stay allocated while the frame extent is unchanged, the nodes queue their
// kernels on the host's stream, and the host synchronises once per frame.
// Ports with several producers in the document are fed by their own edges
// (the reference hands every input port the previous node's buffer).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "../../include/cpipe_b200.h"
#include "host_internal.h"
#include "json_lite.h"

namespace {

using cpb::json::Value;

struct PNode {
    std::string id, type;
    const cpipe_plugin_desc_t* desc = nullptr;
    std::shared_ptr<Value> manifest;
    Value params;
    bool implicit = false;
    std::vector<std::string> in_ports, out_ports;
    std::vector<int> in_src;  // per input port: producing node (planned index), -1 = the pipeline input
    int out_format = 0;
};

struct Edge {
    int from, to;
    std::string from_port, to_port;
};

int format_from_name(const std::string& s) {
    if (s == "R16_UINT") return CPIPE_FMT_R16_UINT;
    if (s == "R32_SFLOAT") return CPIPE_FMT_R32_SFLOAT;
    if (s == "R16G16B16A16_SFLOAT") return CPIPE_FMT_R16G16B16A16_SFLOAT;
    if (s == "R8G8B8A8_UNORM") return CPIPE_FMT_R8G8B8A8_UNORM;
    if (s == "R16G16B16A16_UNORM") return CPIPE_FMT_R16G16B16A16_UNORM;
    return 0;
}

const Value* port_of(const Value& manifest, const char* kind, const std::string& name) {
    const Value* ports = manifest.get("ports");
    if (!ports || !ports->is_arr()) return nullptr;
    for (const Value& p : ports->a)
        if (p.str("kind") == kind && p.str("name") == name) return &p;
    return nullptr;
}
std::vector<std::string> port_names(const Value& manifest, const char* kind) {
    std::vector<std::string> out;
    const Value* ports = manifest.get("ports");
    if (ports && ports->is_arr())
        for (const Value& p : ports->a)
            if (p.str("kind") == kind) out.push_back(p.str("name"));
    return out;
}
struct Caps {
    std::vector<std::string> channels, precisions;
};
Caps caps_of(const Value* port) {
    Caps c;
    const Value* caps = port ? port->get("caps") : nullptr;
    if (caps) {
        c.channels = caps->strings("channels");
        c.precisions = caps->strings("precision");
    }
    return c;
}
std::string format_of_caps(const Caps& c) {
    const bool r = c.channels == std::vector<std::string>{"r"}, rgba = c.channels == std::vector<std::string>{"rgba"};
    if (c.precisions.size() != 1) return "";
    const std::string& p = c.precisions[0];
    if (r && p == "u16") return "R16_UINT";
    if (r && p == "f32") return "R32_SFLOAT";
    if (rgba && p == "f16") return "R16G16B16A16_SFLOAT";
    if (rgba && p == "u8") return "R8G8B8A8_UNORM";
    if (rgba && p == "u16") return "R16G16B16A16_UNORM";
    return "";
}
bool intersects(const std::vector<std::string>& a, const std::vector<std::string>& b) {
    if (a.empty() || b.empty()) return true;
    for (const auto& x : a)
        if (std::find(b.begin(), b.end(), x) != b.end()) return true;
    return false;
}
bool direct_conversion(const std::string& from, const std::string& to) {
    return (from == "R16_UINT" && to == "R32_SFLOAT") || (from == "R32_SFLOAT" && to == "R16G16B16A16_SFLOAT") ||
           (from == "R16G16B16A16_SFLOAT" && to == "R8G8B8A8_UNORM") ||
           (from == "R16G16B16A16_SFLOAT" && to == "R16G16B16A16_UNORM");
}
std::vector<std::string> port_steps(const Value& manifest, const char* kind, const std::string& port, const char* field) {
    const Value* p = port_of(manifest, kind, port);
    const Value* m = p ? p->get("metadata") : nullptr;
    return m ? m->strings(field) : std::vector<std::string>{};
}
std::string color_role(const Value& manifest, const char* field) {
    const Value* c = manifest.get("color");
    return c ? c->str(field, "any") : std::string("any");
}
bool roles_compatible(const std::string& produced, const std::string& required) {
    return produced.empty() || required.empty() || produced == "any" || required == "any" || produced == required;
}

// Pipeline.cpp:214-300: every param must be declared and of its declared type
// (numbers within their range, enums within enum_values).
int check_params(const Value& manifest, const Value& params, std::string* err) {
    if (params.kind == Value::Null) return CPIPE_OK;
    if (!params.is_obj()) {
        *err = "node params must be an object";
        return CPIPE_BAD_INDEX;
    }
    const Value* decls = manifest.get("params");
    for (const auto& kv : params.o) {
        const Value* d = nullptr;
        if (decls && decls->is_arr())
            for (const Value& x : decls->a)
                if (x.str("name") == kv.first) d = &x;
        if (!d) {
            *err = "unknown node param: " + kv.first;
            return CPIPE_BAD_INDEX;
        }
        const std::string type = d->str("type");
        const Value& v = kv.second;
        if (type == "enum") {
            const auto values = d->strings("enum_values");
            if (!v.is_str() || std::find(values.begin(), values.end(), v.s) == values.end()) {
                *err = "node param outside enum: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
        } else if (type == "number") {
            if (!v.is_num()) {
                *err = "node param must be number: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
            const Value* range = d->get("range");
            const Value* lo = range ? range->get("min") : nullptr;
            const Value* hi = range ? range->get("max") : nullptr;
            if ((lo && lo->is_num() && v.n < lo->n) || (hi && hi->is_num() && v.n > hi->n)) {
                *err = "node param outside range: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
        } else if (type == "boolean") {
            if (v.kind != Value::Bool) {
                *err = "node param must be boolean: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
        } else if (type == "string") {
            if (!v.is_str()) {
                *err = "node param must be string: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
        } else if (type == "array") {
            if (!v.is_arr()) {
                *err = "node param must be array: " + kv.first;
                return CPIPE_BAD_INDEX;
            }
        } else {
            *err = "unsupported node param type: " + kv.first;
            return CPIPE_BAD_INDEX;
        }
    }
    return CPIPE_OK;
}

// Kahn's algorithm, ready nodes taken in first-in order; empty when cyclic.
std::vector<int> topo_order(int n, const std::vector<Edge>& edges) {
    std::vector<std::vector<int>> adj(n);
    std::vector<int> indeg(n, 0), order;
    for (const Edge& e : edges) {
        adj[e.from].push_back(e.to);
        ++indeg[e.to];
    }
    std::deque<int> ready;
    for (int i = 0; i < n; ++i)
        if (indeg[i] == 0) ready.push_back(i);
    while (!ready.empty()) {
        const int c = ready.front();
        ready.pop_front();
        order.push_back(c);
        for (int nx : adj[c])
            if (--indeg[nx] == 0) ready.push_back(nx);
    }
    if ((int)order.size() != n) order.clear();
    return order;
}

}  // namespace

namespace {
struct ParamsDeleter {
    void operator()(cpipe_b200_params* p) const { cpipe_b200_params_destroy(p); }
};
}  // namespace

struct cpipe_b200_pipeline {
    cpipe_b200_host* host = nullptr;
    std::string error, input_port;
    int input_format = 0;
    std::vector<PNode> nodes;  // planned, in execution order
    std::vector<std::unique_ptr<cpipe_b200_params, ParamsDeleter>> params;
    // memory plan for the current extent
    uint32_t w = 0, h = 0;
    std::vector<int> slot_of;  // per node
    std::vector<size_t> slot_bytes;
    std::vector<void*> slots;
    uint64_t peak = 0;
    std::vector<cpipe_b200_buffer*> views;  // per node, this run's output handles
};

namespace {

int fail(cpipe_b200_pipeline* p, int status, const std::string& msg) {
    p->error = msg;
    return status;
}

void release_slots(cpipe_b200_pipeline* p) {
    if (!p->slots.empty() && p->host) cudaStreamSynchronize(cpb_host_stream(p->host));
    for (void* s : p->slots) cudaFree(s);
    p->slots.clear();
}
void release_views(cpipe_b200_pipeline* p) {
    for (auto* v : p->views) cpipe_b200_buffer_destroy(v);
    p->views.assign(p->nodes.size(), nullptr);
}

// Live range of node i's output: [i, last consumer] (the last node's output
// stays live to the end); slots by first fit over the execution order.
void plan_memory(cpipe_b200_pipeline* p, uint32_t w, uint32_t h, uint64_t input_bytes) {
    const int n = (int)p->nodes.size();
    std::vector<int> last(n);
    for (int i = 0; i < n; ++i) last[i] = i == n - 1 ? n : i;
    for (int i = 0; i < n; ++i)
        for (int src : p->nodes[i].in_src)
            if (src >= 0) last[src] = std::max(last[src], i);
    p->slot_of.assign(n, -1);
    p->slot_bytes.clear();
    std::vector<std::vector<int>> members;
    for (int i = 0; i < n; ++i) {
        const size_t bytes = (size_t)w * h * cpb_format_bytes(p->nodes[i].out_format);
        int chosen = -1;
        for (int s = 0; s < (int)members.size() && chosen < 0; ++s) {
            bool free = true;
            for (int m : members[s]) free = free && (last[m] < i || m > last[i]);
            if (free) chosen = s;
        }
        if (chosen < 0) {
            chosen = (int)members.size();
            members.emplace_back();
            p->slot_bytes.push_back(0);
        }
        members[chosen].push_back(i);
        p->slot_bytes[chosen] = std::max(p->slot_bytes[chosen], bytes);
        p->slot_of[i] = chosen;
    }
    p->peak = input_bytes;
    for (size_t b : p->slot_bytes) p->peak += b;
}

cpipe_b200_params* make_params(const Value& v) {
    auto* p = cpipe_b200_params_create();
    if (!p || !v.is_obj()) return p;
    for (const auto& kv : v.o) {
        if (kv.second.is_num()) cpipe_b200_params_set_double(p, kv.first.c_str(), kv.second.n);
        else if (kv.second.is_str()) cpipe_b200_params_set_string(p, kv.first.c_str(), kv.second.s.c_str());
        else if (kv.second.kind == Value::Bool) cpipe_b200_params_set_bool(p, kv.first.c_str(), kv.second.b ? 1 : 0);
    }
    return p;
}

int load(cpipe_b200_pipeline* P, const char* text, size_t n, const char* until) {
    Value doc;
    std::string err;
    if (!cpb::json::parse(text, n, &doc, &err)) return fail(P, CPIPE_FAILED, "failed to parse pipeline JSON: " + err);
    if (!doc.is_obj() || doc.str("version") != "0.4")
        return fail(P, CPIPE_FAILED, "schema version mismatch (pipeline documents are version 0.4)");
    const Value* jnodes = doc.get("nodes");
    const Value* jedges = doc.get("edges");
    const Value* jinputs = doc.get("inputs");
    if (!jnodes || !jnodes->is_arr() || !jedges || !jedges->is_arr() || !jinputs || !jinputs->is_arr())
        return fail(P, CPIPE_FAILED, "pipeline schema validation failed: nodes, edges and inputs are required arrays");
    if (jinputs->a.size() != 1)
        return fail(P, CPIPE_UNSUPPORTED, "only one pipeline input is supported");
    const Value& in0 = jinputs->a[0];
    P->input_port = in0.str("port");
    P->input_format = format_from_name(in0.str("format"));
    // document nodes and edges
    std::vector<PNode> doc_nodes;
    std::map<std::string, int> index;
    for (const Value& jn : jnodes->a) {
        if (!jn.is_obj() || !jn.get("id") || !jn.get("id")->is_str() || !jn.get("type") || !jn.get("type")->is_str())
            return fail(P, CPIPE_FAILED, "pipeline schema validation failed: node needs id and type");
        PNode pn;
        pn.id = jn.str("id");
        pn.type = jn.str("type");
        if (const Value* pv = jn.get("params")) pn.params = *pv;
        if (index.count(pn.id)) return fail(P, CPIPE_FAILED, "pipeline schema validation failed: duplicate node id " + pn.id);
        index[pn.id] = (int)doc_nodes.size();
        doc_nodes.push_back(std::move(pn));
    }
    std::vector<Edge> doc_edges;
    for (const Value& je : jedges->a) {
        const std::string from = je.str("from"), to = je.str("to");
        const size_t df = from.find('.'), dt = to.find('.');
        const std::string fn = from.substr(0, df), tn = to.substr(0, dt);
        if (!index.count(fn) || !index.count(tn)) return fail(P, CPIPE_BAD_INDEX, "dangling edge in pipeline");
        doc_edges.push_back(Edge{index[fn], index[tn], df == std::string::npos ? "" : from.substr(df + 1),
                                 dt == std::string::npos ? "" : to.substr(dt + 1)});
    }
    // the nodes to plan: all, or `until` and its ancestors
    std::vector<char> keep(doc_nodes.size(), until ? 0 : 1);
    if (until) {
        if (!index.count(until)) return fail(P, CPIPE_BAD_INDEX, std::string("unknown node id: ") + until);
        std::vector<int> stack{index[until]};
        while (!stack.empty()) {
            const int c = stack.back();
            stack.pop_back();
            if (keep[c]) continue;
            keep[c] = 1;
            for (const Edge& e : doc_edges)
                if (e.to == c) stack.push_back(e.from);
        }
    }
    std::vector<int> remap(doc_nodes.size(), -1);
    std::vector<PNode> nodes;
    for (size_t i = 0; i < doc_nodes.size(); ++i) {
        if (!keep[i]) continue;
        PNode& pn = doc_nodes[i];
        if (pn.type == "com.cpipe.precision_convert") return fail(P, CPIPE_BAD_INDEX, "reserved implicit node type: " + pn.type);
        pn.desc = cpipe_b200_find_node(pn.type.c_str());
        if (!pn.desc) return fail(P, CPIPE_BAD_INDEX, "unknown node type: " + pn.type);
        pn.manifest = std::make_shared<Value>();
        if (!cpb::json::parse(pn.desc->manifest_json, std::strlen(pn.desc->manifest_json), pn.manifest.get(), &err))
            return fail(P, CPIPE_INTERNAL_ERROR, "node manifest does not parse: " + pn.type);
        int st = check_params(*pn.manifest, pn.params, &err);
        if (st != CPIPE_OK) return fail(P, st, err);
        pn.in_ports = port_names(*pn.manifest, "in");
        pn.out_ports = port_names(*pn.manifest, "out");
        remap[i] = (int)nodes.size();
        nodes.push_back(pn);
    }
    std::vector<Edge> edges;
    for (const Edge& e : doc_edges)
        if (keep[e.from] && keep[e.to]) edges.push_back(Edge{remap[e.from], remap[e.to], e.from_port, e.to_port});
    for (const Edge& e : edges) {
        if (!port_of(*nodes[e.from].manifest, "out", e.from_port) || !port_of(*nodes[e.to].manifest, "in", e.to_port))
            return fail(P, CPIPE_BAD_INDEX, "edge names a port the node does not have: " + nodes[e.from].id + "." +
                                                e.from_port + " -> " + nodes[e.to].id + "." + e.to_port);
    }
    const std::vector<int> order = topo_order((int)nodes.size(), edges);
    if (order.size() != nodes.size()) return fail(P, CPIPE_FAILED, "cycle in pipeline graph");
    // steps and colour roles (Pipeline.cpp:469-504)
    std::vector<std::vector<std::string>> steps(nodes.size());
    auto add_unique = [](std::vector<std::string>* v, const std::vector<std::string>& s) {
        for (const auto& x : s)
            if (std::find(v->begin(), v->end(), x) == v->end()) v->push_back(x);
    };
    for (int i : order) {
        for (const Edge& e : edges)
            if (e.to == i) add_unique(&steps[i], steps[e.from]);
        for (const Edge& e : edges)
            if (e.from == i) add_unique(&steps[i], port_steps(*nodes[i].manifest, "out", e.from_port, "sets_steps_applied"));
    }
    for (const Edge& e : edges) {
        for (const auto& s : port_steps(*nodes[e.to].manifest, "in", e.to_port, "requires_steps_applied"))
            if (std::find(steps[e.from].begin(), steps[e.from].end(), s) == steps[e.from].end())
                return fail(P, CPIPE_NEED_METADATA, "metadata step required by pipeline edge is not produced: " + s);
        const std::string a = color_role(*nodes[e.from].manifest, "output_role");
        const std::string b = color_role(*nodes[e.to].manifest, "input_role");
        if (!roles_compatible(a, b)) return fail(P, CPIPE_NEED_METADATA, "color role mismatch on pipeline edge: " + a + " -> " + b);
    }
    // precision planning (PrecisionPlanner::auto_insert)
    const cpipe_plugin_desc_t* pc_desc = cpipe_b200_find_node("com.cpipe.precision_convert");
    std::vector<Edge> planned;
    for (const Edge& e : edges) {
        const Caps produced = caps_of(port_of(*nodes[e.from].manifest, "out", e.from_port));
        const Caps required = caps_of(port_of(*nodes[e.to].manifest, "in", e.to_port));
        if (intersects(produced.precisions, required.precisions)) {
            planned.push_back(e);
            continue;
        }
        const std::string ff = format_of_caps(produced), tf = format_of_caps(required);
        if (ff.empty() || tf.empty() || !direct_conversion(ff, tf) || !pc_desc)
            return fail(P, CPIPE_BAD_PRECISION, "precision mismatch on pipeline edge");
        PNode pc;
        pc.id = "__precision_convert_" + std::to_string(e.from) + "_" + std::to_string(e.to);
        pc.type = "com.cpipe.precision_convert";
        pc.desc = pc_desc;
        pc.manifest = std::make_shared<Value>();
        cpb::json::parse(pc_desc->manifest_json, std::strlen(pc_desc->manifest_json), pc.manifest.get(), &err);
        pc.params.kind = Value::Object;
        Value target;
        target.kind = Value::String;
        target.s = tf;
        pc.params.o.emplace_back("target_format", target);
        pc.implicit = true;
        pc.in_ports = port_names(*pc.manifest, "in");
        pc.out_ports = port_names(*pc.manifest, "out");
        const int k = (int)nodes.size();
        nodes.push_back(pc);
        planned.push_back(Edge{e.from, k, e.from_port, pc.in_ports.empty() ? "in" : pc.in_ports[0]});
        planned.push_back(Edge{k, e.to, pc.out_ports.empty() ? "out" : pc.out_ports[0], e.to_port});
    }
    // Input ports no edge feeds take the pipeline input; one whose precision
    // differs gets an implicit converter too (the reference hands the source's
    // buffer over unchanged and fails in the node).
    {
        std::string in_name;
        switch (P->input_format) {
            case CPIPE_FMT_R16_UINT: in_name = "R16_UINT"; break;
            case CPIPE_FMT_R32_SFLOAT: in_name = "R32_SFLOAT"; break;
            case CPIPE_FMT_R16G16B16A16_SFLOAT: in_name = "R16G16B16A16_SFLOAT"; break;
            default: break;
        }
        const size_t n_doc = nodes.size();
        for (size_t i = 0; i < n_doc && !in_name.empty(); ++i) {
            for (const std::string& port : std::vector<std::string>(nodes[i].in_ports)) {
                bool fed = false;
                for (const Edge& e : planned) fed = fed || (e.to == (int)i && e.to_port == port);
                if (fed) continue;
                const Caps required = caps_of(port_of(*nodes[i].manifest, "in", port));
                const std::string tf = format_of_caps(required);
                const std::string have = in_name == "R16_UINT" ? "u16" : (in_name == "R32_SFLOAT" ? "f32" : "f16");
                if (intersects(std::vector<std::string>{have}, required.precisions)) continue;
                if (tf.empty() || !direct_conversion(in_name, tf) || !pc_desc)
                    return fail(P, CPIPE_BAD_PRECISION, "precision mismatch between the pipeline input and " + nodes[i].id);
                PNode pc;
                pc.id = "__precision_convert_input_" + std::to_string(i);
                pc.type = "com.cpipe.precision_convert";
                pc.desc = pc_desc;
                pc.manifest = std::make_shared<Value>();
                cpb::json::parse(pc_desc->manifest_json, std::strlen(pc_desc->manifest_json), pc.manifest.get(), &err);
                pc.params.kind = Value::Object;
                Value target;
                target.kind = Value::String;
                target.s = tf;
                pc.params.o.emplace_back("target_format", target);
                pc.implicit = true;
                pc.in_ports = port_names(*pc.manifest, "in");
                pc.out_ports = port_names(*pc.manifest, "out");
                const int k = (int)nodes.size();
                nodes.push_back(pc);
                planned.push_back(Edge{k, (int)i, pc.out_ports.empty() ? "out" : pc.out_ports[0], port});
            }
        }
    }
    const std::vector<int> porder = topo_order((int)nodes.size(), planned);
    if (porder.size() != nodes.size()) return fail(P, CPIPE_FAILED, "cycle in precision-planned pipeline graph");
    std::vector<int> pos(nodes.size());
    for (size_t k = 0; k < porder.size(); ++k) pos[porder[k]] = (int)k;
    P->nodes.clear();
    for (int i : porder) P->nodes.push_back(nodes[i]);
    for (auto& pn : P->nodes) pn.in_src.assign(std::max<size_t>(pn.in_ports.size(), 1), -1);
    for (const Edge& e : planned) {
        PNode& to = P->nodes[pos[e.to]];
        const auto it = std::find(to.in_ports.begin(), to.in_ports.end(), e.to_port);
        const size_t slot = it == to.in_ports.end() ? 0 : (size_t)(it - to.in_ports.begin());
        to.in_src[slot] = pos[e.from];
    }
    // output formats (output_layout_for_node, Pipeline.cpp:127-172)
    for (auto& pn : P->nodes) {
        if (pn.out_ports.empty()) return fail(P, CPIPE_UNSUPPORTED, "node without an output port: " + pn.id);
        if (pn.type == "com.cpipe.precision_convert") {
            const Value* t = pn.params.get("target_format");
            pn.out_format = t && t->is_str() ? format_from_name(t->s) : 0;
        } else if (pn.type == "com.cpipe.color.scene_linear_to_display") {
            const Value* t = pn.params.get("target");
            const std::string target = t && t->is_str() ? t->s : "sRGB";
            pn.out_format = target == "sRGB" ? CPIPE_FMT_R8G8B8A8_UNORM
                                             : (target == "BT2020-PQ" ? CPIPE_FMT_R16G16B16A16_UNORM : 0);
        } else {
            pn.out_format = format_from_name(format_of_caps(caps_of(port_of(*pn.manifest, "out", pn.out_ports[0]))));
        }
        if (pn.out_format == 0) return fail(P, CPIPE_FAILED, "unsupported output port format: " + pn.id);
    }
    for (const auto& pn : P->nodes) P->params.emplace_back(make_params(pn.params));
    P->views.assign(P->nodes.size(), nullptr);
    return CPIPE_OK;
}

}  // namespace

extern "C" {

namespace {
thread_local std::string g_load_error;
}

cpipe_b200_pipeline* cpipe_b200_pipeline_load(cpipe_b200_host* host, const char* json, size_t json_bytes,
                                              const char* until, int* status) {
    int st = CPIPE_BAD_INDEX;
    cpipe_b200_pipeline* p = nullptr;
    g_load_error = json ? "" : "no pipeline document";
    if (json) {
        p = new (std::nothrow) cpipe_b200_pipeline();
        if (!p) {
            st = CPIPE_OOM;
        } else {
            p->host = host;
            try {
                st = load(p, json, json_bytes, until);
            } catch (...) {
                st = CPIPE_INTERNAL_ERROR;
                p->error = "pipeline load failed";
            }
            if (st != CPIPE_OK) {
                g_load_error = p->error;
                if (host) cpb_host_set_error(host, p->error);
            }
        }
    }
    if (status) *status = st;
    if (st != CPIPE_OK) {
        delete p;
        return nullptr;
    }
    return p;
}

void cpipe_b200_pipeline_destroy(cpipe_b200_pipeline* p) {
    if (!p) return;
    release_views(p);
    release_slots(p);
    delete p;
}

const char* cpipe_b200_pipeline_last_error(const cpipe_b200_pipeline* p) {
    return p ? p->error.c_str() : g_load_error.c_str();
}
size_t cpipe_b200_pipeline_node_count(const cpipe_b200_pipeline* p) { return p ? p->nodes.size() : 0; }
const char* cpipe_b200_pipeline_node_id(const cpipe_b200_pipeline* p, size_t i) {
    return p && i < p->nodes.size() ? p->nodes[i].id.c_str() : nullptr;
}
const char* cpipe_b200_pipeline_node_type(const cpipe_b200_pipeline* p, size_t i) {
    return p && i < p->nodes.size() ? p->nodes[i].type.c_str() : nullptr;
}

int cpipe_b200_pipeline_memory_plan(cpipe_b200_pipeline* p, uint32_t w, uint32_t h, uint64_t* peak_bytes,
                                    uint32_t* slots) {
    if (!p || w == 0 || h == 0) return CPIPE_BAD_INDEX;
    cpipe_b200_pipeline q;
    q.nodes = p->nodes;
    plan_memory(&q, w, h, (uint64_t)w * h * cpb_format_bytes(p->input_format ? p->input_format : CPIPE_FMT_R16_UINT));
    if (peak_bytes) *peak_bytes = q.peak;
    if (slots) *slots = (uint32_t)q.slot_bytes.size();
    return CPIPE_OK;
}

int cpipe_b200_pipeline_run(cpipe_b200_pipeline* p, cpipe_b200_buffer* input, cpipe_b200_buffer** output) {
    if (!p || !input) return CPIPE_BAD_INDEX;
    if (!p->host) return fail(p, CPIPE_BAD_INDEX, "pipeline loaded without a host (plan only)");
    try {
        uint32_t w = 0, h = 0;
        cpb_buffer_extent(input, &w, &h);
        if (p->input_format && cpb_buffer_format(input) != p->input_format)
            return fail(p, CPIPE_BAD_PRECISION, "input buffer format differs from the pipeline input port " + p->input_port);
        if (w != p->w || h != p->h || p->slots.empty()) {
            release_views(p);
            release_slots(p);
            plan_memory(p, w, h, (uint64_t)w * h * cpb_format_bytes(cpb_buffer_format(input)));
            const uint64_t cap = cpb_host_memory_cap(p->host);
            if (cap && p->peak > cap) return fail(p, CPIPE_OOM, "memory peak exceeds device cap");
            for (size_t b : p->slot_bytes) {
                void* d = nullptr;
                if (cudaMalloc(&d, b) != cudaSuccess) {
                    cudaGetLastError();
                    release_slots(p);
                    return fail(p, CPIPE_OOM, "planner slot allocation failed");
                }
                p->slots.push_back(d);
            }
            p->w = w;
            p->h = h;
        }
        release_views(p);
        for (size_t i = 0; i < p->nodes.size(); ++i) {
            const PNode& pn = p->nodes[i];
            p->views[i] = cpb_buffer_view(p->host, pn.out_format, w, h, p->slots[p->slot_of[i]]);
            if (!p->views[i]) return fail(p, CPIPE_OOM, "buffer handle");
            std::vector<cpipe_b200_buffer*> ins;
            for (int src : pn.in_src) ins.push_back(src < 0 ? input : p->views[src]);
            cpipe_b200_buffer* outs[1] = {p->views[i]};
            const int st = cpb_run_node(p->host, pn.desc, p->params[i].get(), ins.data(), ins.size(), outs, 1, false);
            if (st != CPIPE_OK) {
                cudaStreamSynchronize(cpb_host_stream(p->host));
                return fail(p, st, "node process failed: " + pn.id + ": " + cpb_host_error(p->host));
            }
        }
        const cudaError_t e = cudaStreamSynchronize(cpb_host_stream(p->host));
        if (e != cudaSuccess) return fail(p, CPIPE_INTERNAL_ERROR, cudaGetErrorString(e));
        if (output) *output = p->views.back();
        p->error.clear();
        return CPIPE_OK;
    } catch (...) {
        return fail(p, CPIPE_INTERNAL_ERROR, "pipeline run failed");
    }
}

}  // extern "C"
