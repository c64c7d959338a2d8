// mesh_order.cpp - node renumbering for gather locality (host code).
//
// The element pass reads the coordinates and increments of every element's
// nodes through the connectivity, so nodes that share elements should sit
// close together in the node arrays: consecutive elements then touch the same
// few cache lines.  Meshes from DynELA scripts keep the numbering of their
// createNode calls (DynELA::createNode, DynELA.C:160-200), which the element
// pass has to live with unless the engine renumbers its own copy of the nodes.
//
// The ordering is reverse Cuthill-McKee on the node graph (two nodes are
// adjacent when an element holds both): breadth-first levels from a
// pseudo-peripheral node (George and Liu's iteration: restart from a node of
// least degree in the last level while the eccentricity grows), the
// unnumbered neighbours of each node taken by increasing degree, the whole
// sequence reversed.  Degrees count distinct neighbours.  Disconnected parts
// are numbered one after another, each from its own pseudo-peripheral node.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "dnlgpu.h"

namespace
{
struct NodeGraph
{
  int n;
  std::vector<int> off, elems; // node -> incident elements
  std::vector<int> degree;     // distinct neighbours
  const int32_t *conn;
  int npe;

  NodeGraph(int nN, int nE, int npe_, const int32_t *conn_) : n(nN), off(nN + 1, 0), degree(nN, 0), conn(conn_), npe(npe_)
  {
    const long long nIP = (long long)nE * npe;
    for (long long k = 0; k < nIP; k++)
      off[conn[k] + 1]++;
    for (int i = 0; i < nN; i++)
      off[i + 1] += off[i];
    elems.resize(nIP);
    std::vector<int> cur(off.begin(), off.end() - 1);
    for (long long k = 0; k < nIP; k++)
      elems[cur[conn[k]]++] = (int)(k / npe);
    std::vector<int> mark(nN, -1);
    for (int v = 0; v < nN; v++)
    {
      mark[v] = v;
      int d = 0;
      for (int j = off[v]; j < off[v + 1]; j++)
        for (int l = 0; l < npe; l++)
        {
          const int u = conn[(size_t)elems[j] * npe + l];
          if (mark[u] != v)
          {
            mark[u] = v;
            d++;
          }
        }
      degree[v] = d;
    }
  }

  // calls f(u) once for each neighbour u of v (mark: scratch, stamp: unique per call)
  template <class F> void neighbours(int v, std::vector<int> &mark, int stamp, F f) const
  {
    mark[v] = stamp;
    for (int j = off[v]; j < off[v + 1]; j++)
      for (int l = 0; l < npe; l++)
      {
        const int u = conn[(size_t)elems[j] * npe + l];
        if (mark[u] != stamp)
        {
          mark[u] = stamp;
          f(u);
        }
      }
  }
};

// Breadth-first levels from r over the nodes not yet numbered: the number of
// levels and, in `last`, the nodes of the last one.
int bfs_levels(const NodeGraph &G, int r, const std::vector<char> &numbered, std::vector<int> &level,
               std::vector<int> &queue, std::vector<int> &last)
{
  queue.clear();
  queue.push_back(r);
  level[r] = 0;
  int depth = 0;
  for (size_t h = 0; h < queue.size(); h++)
  {
    const int v = queue[h];
    for (int j = G.off[v]; j < G.off[v + 1]; j++)
      for (int l = 0; l < G.npe; l++)
      {
        const int u = G.conn[(size_t)G.elems[j] * G.npe + l];
        if (!numbered[u] && level[u] < 0)
        {
          level[u] = level[v] + 1;
          depth = std::max(depth, level[u]);
          queue.push_back(u);
        }
      }
  }
  last.clear();
  for (int v : queue)
    if (level[v] == depth)
      last.push_back(v);
  for (int v : queue)
    level[v] = -1;
  return depth;
}
} // namespace

int dnl_mesh_order_rcm(int32_t n_nodes, int32_t n_elems, int32_t npe, const int32_t *conn, int32_t *order)
{
  if (n_nodes < 0 || n_elems < 0 || (npe != 4 && npe != 8) || !order || (n_elems > 0 && !conn))
    return DNL_ERR_ARG;
  for (long long k = 0; k < (long long)n_elems * npe; k++)
    if (conn[k] < 0 || conn[k] >= n_nodes)
      return DNL_ERR_ARG;
  const NodeGraph G(n_nodes, n_elems, npe, conn);
  std::vector<char> numbered(n_nodes, 0);
  std::vector<int> level(n_nodes, -1), queue, last, mark(n_nodes, -1), cand;
  std::vector<int> seq;
  seq.reserve(n_nodes);
  int stamp = 0;
  for (int s = 0; s < n_nodes; s++)
  {
    if (numbered[s])
      continue;
    // pseudo-peripheral node of s's part
    int r = s, ecc = bfs_levels(G, r, numbered, level, queue, last);
    for (int it = 0; it < 16; it++)
    {
      int x = last[0];
      for (int v : last)
        if (G.degree[v] < G.degree[x] || (G.degree[v] == G.degree[x] && v < x))
          x = v;
      std::vector<int> lastX;
      const int ex = bfs_levels(G, x, numbered, level, queue, lastX);
      if (ex <= ecc)
        break;
      r = x;
      ecc = ex;
      last.swap(lastX);
    }
    // Cuthill-McKee from r
    size_t h = seq.size();
    seq.push_back(r);
    numbered[r] = 1;
    for (; h < seq.size(); h++)
    {
      cand.clear();
      G.neighbours(seq[h], mark, stamp++, [&](int u) {
        if (!numbered[u])
          cand.push_back(u);
      });
      std::sort(cand.begin(), cand.end(), [&](int a, int b) {
        return G.degree[a] != G.degree[b] ? G.degree[a] < G.degree[b] : a < b;
      });
      for (int u : cand)
      {
        numbered[u] = 1;
        seq.push_back(u);
      }
    }
  }
  for (int k = 0; k < n_nodes; k++)
    order[k] = seq[n_nodes - 1 - k];
  return DNL_OK;
}

int dnl_mesh_span(int32_t n_nodes, int32_t n_elems, int32_t npe, const int32_t *conn, const int32_t *order,
                  double *mean_span)
{
  if (n_nodes < 0 || n_elems < 0 || npe <= 0 || !mean_span || (n_elems > 0 && !conn))
    return DNL_ERR_ARG;
  std::vector<int> rank;
  if (order)
  {
    rank.assign(n_nodes, -1);
    for (int k = 0; k < n_nodes; k++)
    {
      if (order[k] < 0 || order[k] >= n_nodes || rank[order[k]] >= 0)
        return DNL_ERR_ARG;
      rank[order[k]] = k;
    }
  }
  double sum = 0.0;
  for (int e = 0; e < n_elems; e++)
  {
    int lo = 0x7fffffff, hi = -1;
    for (int l = 0; l < npe; l++)
    {
      const int v = conn[(size_t)e * npe + l];
      if (v < 0 || v >= n_nodes)
        return DNL_ERR_ARG;
      const int r = order ? rank[v] : v;
      lo = std::min(lo, r);
      hi = std::max(hi, r);
    }
    sum += hi - lo;
  }
  *mean_span = n_elems > 0 ? sum / n_elems : 0.0;
  return DNL_OK;
}
