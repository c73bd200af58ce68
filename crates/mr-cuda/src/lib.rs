//! `CudaIsolatedProvider`: NegotiatedRouter's "route each net alone" batch on a
//! B200, through the C ABI of libmr_cuda.so (`include/mr_cuda.h`).
//!
//! The seam is `mr_cpu::IsolatedRouteProvider`
//! (crates/mr-cpu/src/negotiated.rs:554-560), the one the Metal adapter
//! implements (crates/mr-cli/src/lib.rs:612-625).  The library solves every
//! window, retries on the whole board only the nets unreachable in their window
//! (the adapter's rule, crates/mr-cli/src/lib.rs:574-607) and returns the
//! canonical `(cost, hops, lower predecessor)` path of every net, aligned with
//! `request.nets`, or an error and nothing else.  Any error makes the router
//! rerun the whole batch on the CPU (negotiated.rs:1431-1453).
//!
//! Not buildable in the image the engine was developed in (no Rust toolchain);
//! `Cargo.toml` says how to build it inside the metalroute workspace.

use mr_core::{CellIdx, RouterError};
use mr_cpu::{IsolatedRouteProvider, IsolatedRouteRequest};
use std::ffi::CStr;
use std::os::raw::{c_char, c_int, c_void};

/// `mrc_grid`: the board.  Null masks are absent masks.
#[repr(C)]
struct MrcGrid {
    w: u32,
    h: u32,
    layers: u32,
    cost: *const u32,
    board_constraint: *const u8,
    via_forbidden: *const u8,
}

/// `mrc_net`: endpoints and the net's own (via) pads, any order.
#[repr(C)]
struct MrcNet {
    src: u32,
    dst: u32,
    passable_pads: *const u32,
    n_passable_pads: u32,
    via_passable_pads: *const u32,
    n_via_passable_pads: u32,
}

/// `mrc_window`: inclusive planar rectangle, every layer.
#[repr(C)]
#[derive(Clone, Copy)]
struct MrcWindow {
    x0: u32,
    y0: u32,
    x1: u32,
    y1: u32,
}

/// `mrc_edges`: the already-rounded edge vectors; `Option<Cost>` vias are split
/// into a price and an allowed byte, as mr-metal does (metal/src/lib.rs:484-493).
#[repr(C)]
struct MrcEdges {
    x_edge_costs: *const u32,
    n_x_edge_costs: u32,
    y_edge_costs: *const u32,
    n_y_edge_costs: u32,
    via_edge_costs: *const u32,
    via_allowed: *const u8,
    n_via_edge_costs: u32,
    directed_in_costs: *const u32,
}

/// `mrc_isolated_request`: IsolatedRouteRequest field for field.
#[repr(C)]
struct MrcRequest {
    grid: *const MrcGrid,
    nets: *const MrcNet,
    n_nets: u32,
    windows: *const MrcWindow,
    edges: MrcEdges,
}

const MRC_FLAG_RETRY_FULL: u32 = 0x1;
const MRC_FLAG_NO_WAIT: u32 = 0x4;
const MRC_ERR_BUSY: c_int = 5;
const MRC_NO_PATH: u32 = u32::MAX;

#[link(name = "mr_cuda")]
extern "C" {
    fn mrc_context_create(device: c_int, out: *mut *mut c_void) -> c_int;
    fn mrc_context_destroy(ctx: *mut c_void);
    fn mrc_last_error(ctx: *const c_void) -> *const c_char;
    fn mrc_route_isolated_batch(ctx: *mut c_void, req: *const MrcRequest, flags: u32, out: *mut *mut c_void) -> c_int;
    fn mrc_result_count(r: *const c_void) -> u32;
    fn mrc_result_path_offsets(r: *const c_void) -> *const u64;
    fn mrc_result_path_cells(r: *const c_void) -> *const u32;
    fn mrc_result_search_costs(r: *const c_void) -> *const u32;
    fn mrc_result_free(r: *mut c_void);
}

/// One CUDA context of the engine; calls on it serialise inside the library.
pub struct CudaIsolatedProvider {
    ctx: *mut c_void,
    /// Fail at once when another thread holds the context (the Metal adapter's
    /// try_lock, crates/mr-cli/src/lib.rs:620-622); the router then takes its
    /// CPU path.  `false` waits for the context instead.
    pub no_wait: bool,
}

// The context is thread-safe: the library serialises calls on it.
unsafe impl Send for CudaIsolatedProvider {}
unsafe impl Sync for CudaIsolatedProvider {}

impl CudaIsolatedProvider {
    /// A context on CUDA device `device`; `BackendUnavailable` without one.
    pub fn new(device: i32) -> Result<Self, RouterError> {
        let mut ctx = std::ptr::null_mut();
        match unsafe { mrc_context_create(device, &mut ctx) } {
            0 => Ok(Self { ctx, no_wait: true }),
            _ => Err(RouterError::BackendUnavailable(last_error(std::ptr::null()))),
        }
    }
}

impl Drop for CudaIsolatedProvider {
    fn drop(&mut self) {
        unsafe { mrc_context_destroy(self.ctx) }
    }
}

fn last_error(ctx: *const c_void) -> String {
    let p = unsafe { mrc_last_error(ctx) };
    if p.is_null() {
        return "mr-cuda: unknown error".into();
    }
    unsafe { CStr::from_ptr(p) }.to_string_lossy().into_owned()
}

fn or_null<T>(v: &[T]) -> *const T {
    if v.is_empty() {
        std::ptr::null()
    } else {
        v.as_ptr()
    }
}

impl IsolatedRouteProvider for CudaIsolatedProvider {
    fn route_isolated_batch(
        &self,
        request: IsolatedRouteRequest<'_>,
    ) -> Result<Vec<Option<Vec<CellIdx>>>, RouterError> {
        let g = request.grid;
        // Grid::via_forbidden is Vec<bool>: one byte per cell, 0 or 1.
        let grid = MrcGrid {
            w: g.dims.w,
            h: g.dims.h,
            layers: g.dims.layers,
            cost: g.cost.as_ptr(),
            board_constraint: or_null(&g.board_constraint),
            via_forbidden: or_null(&g.via_forbidden) as *const u8,
        };
        let nets: Vec<MrcNet> = request
            .nets
            .iter()
            .map(|n| MrcNet {
                src: n.src,
                dst: n.dst,
                passable_pads: or_null(&n.passable_pads),
                n_passable_pads: n.passable_pads.len() as u32,
                via_passable_pads: or_null(&n.via_passable_pads),
                n_via_passable_pads: n.via_passable_pads.len() as u32,
            })
            .collect();
        let windows: Vec<MrcWindow> = request
            .windows
            .iter()
            .map(|w| MrcWindow { x0: w.x0, y0: w.y0, x1: w.x1, y1: w.y1 })
            .collect();
        let via_costs: Vec<u32> = request.via_edge_costs.iter().map(|v| v.unwrap_or(0)).collect();
        let via_allowed: Vec<u8> = request.via_edge_costs.iter().map(|v| v.is_some() as u8).collect();
        let req = MrcRequest {
            grid: &grid,
            nets: or_null(&nets),
            n_nets: nets.len() as u32,
            windows: or_null(&windows),
            edges: MrcEdges {
                x_edge_costs: or_null(request.x_edge_costs),
                n_x_edge_costs: request.x_edge_costs.len() as u32,
                y_edge_costs: or_null(request.y_edge_costs),
                n_y_edge_costs: request.y_edge_costs.len() as u32,
                via_edge_costs: or_null(&via_costs),
                via_allowed: or_null(&via_allowed),
                n_via_edge_costs: via_costs.len() as u32,
                directed_in_costs: std::ptr::null(),
            },
        };
        let flags = MRC_FLAG_RETRY_FULL | if self.no_wait { MRC_FLAG_NO_WAIT } else { 0 };
        let mut res = std::ptr::null_mut();
        let st = unsafe { mrc_route_isolated_batch(self.ctx, &req, flags, &mut res) };
        if st != 0 {
            let msg = last_error(self.ctx);
            return Err(RouterError::BackendUnavailable(if st == MRC_ERR_BUSY {
                format!("mr-cuda busy: {msg}")
            } else {
                msg
            }));
        }
        // CSR: path i is cells[offsets[i]..offsets[i+1]], empty when unreachable
        let n = unsafe { mrc_result_count(res) } as usize;
        let out = if n != nets.len() {
            Err(RouterError::BackendUnavailable("mr-cuda result is not net-aligned".into()))
        } else {
            let offsets = unsafe { std::slice::from_raw_parts(mrc_result_path_offsets(res), n + 1) };
            let total = offsets[n] as usize;
            let cells: &[u32] = if total == 0 {
                &[]
            } else {
                unsafe { std::slice::from_raw_parts(mrc_result_path_cells(res), total) }
            };
            let costs: &[u32] = if n == 0 {
                &[]
            } else {
                unsafe { std::slice::from_raw_parts(mrc_result_search_costs(res), n) }
            };
            Ok((0..n)
                .map(|i| {
                    (costs[i] != MRC_NO_PATH).then(|| cells[offsets[i] as usize..offsets[i + 1] as usize].to_vec())
                })
                .collect())
        };
        unsafe { mrc_result_free(res) };
        out
    }
}
