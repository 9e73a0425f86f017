// A batch of independent problems as one context: the parts' meshes are laid
// side by side (elements, faces and nodes renumbered with offsets), so every
// residual, Jacobian, SpMV and preconditioner launch covers all problems at
// once, whatever their mesh sizes. The reference solves such problems one at
// a time; the discretization of each part is unchanged: faces never join
// two parts, the Jacobian is block diagonal by part, and each element
// carries its part's Burgers coefficients (mu, a, b). Interior faces of all
// parts come first, then all boundary faces, each part in its own order, so
// each part's tabulated boundary data is a contiguous slice of the batch's.
#include <cstring>
#include <vector>

#include "icx_internal.h"

extern "C" {

icx_status icx_batch_create(icx_ctx** out, int device, int n_parts, icx_ctx* const* parts) {
  if (!out || n_parts < 1 || !parts) return ICX_ERR_INVALID;
  *out = nullptr;
  const icx_ctx* p0 = parts[0];
  for (int k = 0; k < n_parts; ++k) {
    const icx_ctx* q = parts[k];
    if (!q || !q->ready || !q->parts.empty()) return ICX_ERR_INVALID;
    if (q->phys.spacetime) return ICX_ERR_UNSUPPORTED;
    if (q->basis != p0->basis) return ICX_ERR_INVALID;
    if (q->p != p0->p || q->geo_order != p0->geo_order || q->phys.pde != p0->phys.pde ||
        q->phys.interior_penalty != p0->phys.interior_penalty || q->phys.sigma_ic != p0->phys.sigma_ic ||
        q->device != device)
      return ICX_ERR_INVALID;
    if (q->phys.pde == ICX_PDE_NAVIER_STOKES &&
        (q->phys.gamma != p0->phys.gamma || q->phys.Pr != p0->phys.Pr || q->phys.ns_mu != p0->phys.ns_mu ||
         q->conv_flux != p0->conv_flux || q->phys.ns_visc != p0->phys.ns_visc ||
         q->phys.suth[0] != p0->phys.suth[0] || q->phys.suth[1] != p0->phys.suth[1] ||
         q->phys.suth[2] != p0->phys.suth[2]))
      return ICX_ERR_INVALID;
  }
  icx_ctx* c = nullptr;
  icx_status st = icx_create(&c, device);
  if (st != ICX_OK) return st;
  c->p = p0->p;
  c->basis = p0->basis;
  c->geo_order = p0->geo_order;
  c->phys = p0->phys;
  c->conv_flux = p0->conv_flux;
  std::memcpy(c->bctype, p0->bctype, sizeof(c->bctype));
  std::memcpy(c->bcflag, p0->bcflag, sizeof(c->bcflag));
  std::vector<int> node_off(n_parts), el_off(n_parts);
  int nn = 0, ne = 0;
  for (int k = 0; k < n_parts; ++k) {
    node_off[k] = nn;
    el_off[k] = ne;
    nn += (int)(parts[k]->coord.size() / 2);
    ne += parts[k]->n_elem;
  }
  for (int k = 0; k < n_parts; ++k) {
    const icx_ctx* q = parts[k];
    c->coord.insert(c->coord.end(), q->coord.begin(), q->coord.end());
    for (int v : q->el_nodes) c->el_nodes.push_back(v + node_off[k]);
    c->el_level.insert(c->el_level.end(), q->el_level.begin(), q->el_level.end());
    c->el_i.insert(c->el_i.end(), q->el_i.begin(), q->el_i.end());
    c->el_j.insert(c->el_j.end(), q->el_j.begin(), q->el_j.end());
    c->el_grid.insert(c->el_grid.end(), q->n_elem, k);
    if (q->phys.pde == ICX_PDE_BURGERS)
      for (int e = 0; e < q->n_elem; ++e) {
        const double v[5] = {q->phys.mu, q->phys.a[0], q->phys.a[1], q->phys.b[0], q->phys.b[1]};
        c->el_par.insert(c->el_par.end(), v, v + 5);
      }
  }
  // interior faces of every part, then the boundary faces of every part
  for (int pass = 0; pass < 2; ++pass) {
    for (int k = 0; k < n_parts; ++k) {
      const icx_ctx* q = parts[k];
      const int nf = (int)q->faces.size() / 7;
      const int f0 = pass == 0 ? 0 : q->n_interior, f1 = pass == 0 ? q->n_interior : nf;
      for (int f = f0; f < f1; ++f) {
        int rec[7];
        std::memcpy(rec, &q->faces[7 * f], sizeof(rec));
        rec[0] += el_off[k];
        if (rec[1] >= 0) rec[1] += el_off[k];
        c->faces.insert(c->faces.end(), rec, rec + 7);
      }
    }
    if (pass == 0) c->n_interior = (int)c->faces.size() / 7;
  }
  c->n_elem = ne;
  c->nx = c->ny = 0;  // not one grid
  c->parts.assign(parts, parts + n_parts);
  c->has_mesh = c->has_space = c->has_disc = true;
  st = icx_setup(c);
  if (st != ICX_OK) {
    icx_destroy(c);
    return st;
  }
  *out = c;
  return ICX_OK;
}

icx_status icx_batch_offsets(const icx_ctx* c, int* elem_offsets) {
  if (!c || c->parts.empty() || !elem_offsets) return ICX_ERR_INVALID;
  int off = 0;
  for (size_t k = 0; k < c->parts.size(); ++k) {
    elem_offsets[k] = off;
    off += c->parts[k]->n_elem;
  }
  elem_offsets[c->parts.size()] = off;
  return ICX_OK;
}

}  // extern "C"
