//! The isolated-provider contract of NegotiatedRouter, run with the CUDA
//! provider: with the provider, every route equals the CPU route bit for bit
//! (the provider's paths are the CPU's canonical paths), the provider is
//! called once per public route, and the cases where the Metal backend had to
//! fail closed (static via masks, exact board masks) succeed here.
//!
//! The same contract is checked through the C ABI from Python in
//! tests/test_gpu_provider_contract.py (this image has no Rust toolchain).
//! Each test returns early, with a note, on a machine without a CUDA device.

use mr_core::{Dims, Grid, GridCoords, NetEndpoints, ViaModel, OBSTACLE};
use mr_cpu::{IsolatedRouteProvider, IsolatedRouteRequest, NegotiatedRouter};
use mr_cuda::CudaIsolatedProvider;
use std::sync::atomic::{AtomicUsize, Ordering};

/// Counts the calls and whether each one succeeded.
struct Counting {
    inner: CudaIsolatedProvider,
    calls: AtomicUsize,
    ok: AtomicUsize,
}

impl IsolatedRouteProvider for Counting {
    fn route_isolated_batch(
        &self,
        request: IsolatedRouteRequest<'_>,
    ) -> Result<Vec<Option<Vec<mr_core::CellIdx>>>, mr_core::RouterError> {
        self.calls.fetch_add(1, Ordering::Relaxed);
        let r = self.inner.route_isolated_batch(request);
        if r.is_ok() {
            self.ok.fetch_add(1, Ordering::Relaxed);
        }
        r
    }
}

fn provider() -> Option<Counting> {
    match CudaIsolatedProvider::new(0) {
        Ok(mut p) => {
            p.no_wait = false; // tests may run on several threads
            Some(Counting { inner: p, calls: AtomicUsize::new(0), ok: AtomicUsize::new(0) })
        }
        Err(e) => {
            eprintln!("skipped: {e}");
            None
        }
    }
}

fn net(name: &str, src: u32, dst: u32) -> NetEndpoints {
    NetEndpoints { net: name.into(), src, dst, passable_pads: Vec::new(), via_passable_pads: Vec::new() }
}

#[test]
fn reachable_unreachable_and_zero_hop_nets_match_the_cpu() {
    let Some(p) = provider() else { return };
    let dims = Dims::new(5, 5);
    let mut grid = Grid::filled(dims, 1);
    for (x, y) in [(2, 1), (1, 2), (3, 2), (2, 3)] {
        grid.set(dims.idx(x, y), OBSTACLE);
    }
    let nets = vec![
        net("open", dims.idx(0, 4), dims.idx(4, 4)),
        net("blocked", dims.idx(0, 0), dims.idx(2, 2)),
        net("zero", dims.idx(4, 0), dims.idx(4, 0)),
    ];
    let router = NegotiatedRouter::new();
    let cpu = router.route_with_outcome(&grid, &nets).unwrap();
    let gpu = router.route_with_isolated_provider(&grid, &nets, &p).unwrap();
    assert_eq!(gpu, cpu);
    assert_eq!(gpu.alone_routable, [true, false, true]);
    assert_eq!(p.calls.load(Ordering::Relaxed), 1, "one batch per public route");
    assert_eq!(p.ok.load(Ordering::Relaxed), 1, "the provider's batch was accepted");
}

#[test]
fn exact_short_coordinate_and_via_vectors_route_like_the_cpu() {
    let Some(p) = provider() else { return };
    let dims = Dims::with_layers(4, 3, 3);
    let grid = Grid::filled(dims, 1);
    let nets = vec![net("n", dims.idx3(0, 0, 0), dims.idx3(3, 2, 0))];
    let router = NegotiatedRouter::new()
        .with_coords(GridCoords::from_lines(vec![10.0], Vec::new()))
        .with_via_model(ViaModel::with_allowed_steps(3, 7, vec![(0, 1)]));
    let cpu = router.route_with_outcome(&grid, &nets).unwrap();
    let gpu = router.route_with_isolated_provider(&grid, &nets, &p).unwrap();
    assert_eq!(gpu, cpu);
    assert_eq!(p.ok.load(Ordering::Relaxed), 1);
}

#[test]
fn weighted_board_with_static_via_and_board_masks_needs_no_cpu_fallback() {
    let Some(p) = provider() else { return };
    let dims = Dims::with_layers(9, 7, 3);
    let coords = GridCoords::from_lines(
        vec![0.0, 0.2, 0.7, 1.9, 2.0, 4.5, 4.7, 8.0, 8.1],
        vec![0.0, 0.1, 1.0, 1.0, 2.7, 6.0, 6.2],
    );
    let mut grid = Grid::filled(dims, 1);
    grid.set(dims.idx3(2, 3, 0), 0);
    grid.set(dims.idx3(3, 3, 1), 7);
    for (x, y, l) in [(0, 0, 0), (8, 0, 2), (4, 3, 0), (4, 3, 1)] {
        grid.set(dims.idx3(x, y, l), OBSTACLE);
    }
    let own = NetEndpoints {
        passable_pads: vec![dims.idx3(0, 0, 0), dims.idx3(8, 0, 2)],
        ..net("own-pads", dims.idx3(0, 0, 0), dims.idx3(8, 0, 2))
    };
    let nets = vec![
        net("weighted", dims.idx3(0, 3, 0), dims.idx3(8, 3, 2)),
        own,
        net("zero-length", dims.idx3(2, 3, 0), dims.idx3(2, 3, 0)),
    ];
    let router = NegotiatedRouter::new()
        .with_coords(coords)
        .with_via_model(ViaModel::with_allowed_steps(3, 37, vec![(0, 1), (1, 2)]));

    let mut masked = grid.clone();
    masked.via_forbidden = vec![false; dims.len()];
    let mut outlined = grid.clone();
    outlined.board_constraint = vec![0; dims.len()];
    outlined.board_constraint[dims.idx3(1, 1, 0) as usize] |= Grid::BOARD_EDGE_POS_X;

    for (k, g) in [grid, masked, outlined].iter().enumerate() {
        let cpu = router.route_with_outcome(g, &nets).unwrap();
        let gpu = router.route_with_isolated_provider(g, &nets, &p).unwrap();
        assert_eq!(gpu, cpu, "variant {k}");
        assert_eq!(p.ok.load(Ordering::Relaxed), k + 1, "variant {k}: the CUDA batch was accepted");
    }
}
