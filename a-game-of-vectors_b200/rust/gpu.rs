//! gpu.rs — the reference crate's query API on one B200, over the C ABI of include/sieve_gpu.h.
//!
//! Dropped into the reference crate as `src/gpu.rs` (with `pub mod gpu;` in `src/lib.rs` and the
//! link lines of build.rs below), it gives `gpu::Index` the methods of `ivf::Index` the query
//! path uses, with the same signatures: `search(&self, &Corpus, q768, q256, &Params,
//! &mut Scratch, &mut Timing) -> Vec<(f32, u32)>` (src/ivf.rs:621-623), `search_view`,
//! `candidates` and `rerank` (src/ivf.rs:647-815), and `Scratch::new` per worker thread
//! (src/ivf.rs:497-513). Callers written against `ivf::Index` switch by changing the type they
//! open. The corpus lives on the GPU with the index (uploaded by `open`), so the `&Corpus`
//! argument is only checked against the one the index was opened with.
//!
//! `gpu::Scratch` is one sg_context: a stream, device scratch and captured CUDA graphs of its
//! own, so rayon workers that each hold one search the shared index concurrently and overlap on
//! the GPU (the reference's one-Scratch-per-worker pattern, src/bin/search.rs:312-323).
//!
//! build.rs of the reference crate:
//!     println!("cargo:rustc-link-search=native=<repo>/a-game-of-vectors_b200/sieve_gpu/_lib");
//!     println!("cargo:rustc-link-lib=dylib=sieve_gpu");
//!
//! This file is not compiled here: the image that builds the GPU library has no Rust toolchain.
use std::ffi::{CStr, CString, c_char, c_int};
use std::path::Path;

use crate::ivf::{Corpus, Params, Rerank, Timing, View};

#[repr(C)]
#[derive(Default, Clone, Copy)]
struct SgParams {
    nprobe: u32,
    cand: u32,
    rerank_kind: u32,
    rerank_r: u32,
    k: u32,
    has_prune: u32,
    prune_m: u32,
    prune_w: f32,
    has_margin: u32,
    margin: f32,
    has_budget: u32,
    reserved: u32,
    budget: u64,
}

#[repr(C)]
#[derive(Default, Clone, Copy)]
struct SgTiming {
    route: u64,
    scan: u64,
    rerank: u64,
    tier2: u64,
    scanned: u64,
    reranked: u64,
    probed: u64,
    fetch: u64,
    wait: u64,
}

#[repr(C)]
struct SgIndex {
    _opaque: [u8; 0],
}

#[repr(C)]
struct SgContext {
    _opaque: [u8; 0],
}

unsafe extern "C" {
    fn sg_open_ivf(ingest: *const c_char, index: *const c_char, device: c_int, out: *mut *mut SgIndex) -> c_int;
    fn sg_close(ix: *mut SgIndex) -> c_int;
    fn sg_index_info(ix: *const SgIndex, k: *mut u32, n: *mut u64, nblocks: *mut u64, has_t2: *mut u32) -> c_int;
    fn sg_context_open(ix: *mut SgIndex, out: *mut *mut SgContext) -> c_int;
    fn sg_context_close(c: *mut SgContext) -> c_int;
    fn sg_search_ctx(c: *mut SgContext, nq: u32, q768: *const f32, q256: *const f32, p: *const SgParams,
                     allow: *const u64, allow_words: u64, out_scores: *mut f32, out_ids: *mut u32,
                     out_counts: *mut u32, t: *mut SgTiming) -> c_int;
    fn sg_candidates_probes(ix: *mut SgIndex, nq: u32, q256: *const f32, probe_scores: *const f32,
                            probe_clusters: *const u32, probe_counts: *const u32, p: *const SgParams,
                            allow: *const u64, allow_words: u64, out_est: *mut f32, out_ids: *mut u32,
                            out_err: *mut f32, out_counts: *mut u32) -> c_int;
    fn sg_rerank(ix: *mut SgIndex, nq: u32, q768: *const f32, q256: *const f32, est: *const f32,
                 ids: *const u32, err: *const f32, counts: *const u32, stride: u32, p: *const SgParams,
                 out_scores: *mut f32, out_ids: *mut u32, out_counts: *mut u32) -> c_int;
    fn sg_last_error() -> *const c_char;
}

impl From<&Params> for SgParams {
    fn from(p: &Params) -> Self {
        let (kind, r) = match p.rerank {
            Rerank::None => (0, 0),
            Rerank::Prefix => (1, 0),
            Rerank::Full => (2, 0),
            Rerank::Tiered(r) => (3, r),
            Rerank::Ssd(r) => (4, r),
        };
        let mut s = SgParams { nprobe: p.nprobe as u32, cand: p.cand as u32, rerank_kind: kind, rerank_r: r as u32,
                               k: p.k as u32, ..Default::default() };
        if let Some((m, w)) = p.prune {
            (s.has_prune, s.prune_m, s.prune_w) = (1, m as u32, w);
        }
        if let Some(m) = p.margin {
            (s.has_margin, s.margin) = (1, m);
        }
        if let Some(b) = p.budget {
            (s.has_budget, s.budget) = (1, b as u64);
        }
        s
    }
}

fn check(rc: c_int) -> anyhow::Result<()> {
    if rc == 0 {
        return Ok(());
    }
    let msg = unsafe { CStr::from_ptr(sg_last_error()) }.to_string_lossy().into_owned();
    anyhow::bail!("sieve_gpu status {rc}: {msg}")
}

fn add(t: &mut Timing, s: &SgTiming) {
    t.route += s.route;
    t.scan += s.scan;
    t.rerank += s.rerank;
    t.tier2 += s.tier2;
    t.scanned += s.scanned;
    t.reranked += s.reranked;
    t.probed += s.probed;
}

/// An IVF index and its corpus resident on one GPU.
pub struct Index {
    h: *mut SgIndex,
    pub k: usize,
    rows: usize,
}

// The library serialises calls on an index's default context and gives each Scratch its own.
unsafe impl Send for Index {}
unsafe impl Sync for Index {}

impl Index {
    /// `Corpus::open(ingest)` + `Index::open(index)` (src/ivf.rs:75-90, :553-578) onto `device`.
    pub fn open(ingest: &Path, index: &Path, device: i32) -> anyhow::Result<Self> {
        let i = CString::new(ingest.to_str().unwrap())?;
        let x = CString::new(index.to_str().unwrap())?;
        let mut h = std::ptr::null_mut();
        check(unsafe { sg_open_ivf(i.as_ptr(), x.as_ptr(), device, &mut h) })?;
        let (mut k, mut n, mut nb, mut t2) = (0u32, 0u64, 0u64, 0u32);
        check(unsafe { sg_index_info(h, &mut k, &mut n, &mut nb, &mut t2) })?;
        Ok(Self { h, k: k as usize, rows: n as usize })
    }

    /// `Index::search` (src/ivf.rs:621-623): (score, row) best first, ties by ascending row.
    pub fn search(&self, corpus: &Corpus, q768: &[f32], q256: &[f32], p: &Params, s: &mut Scratch,
                  t: &mut Timing) -> Vec<(f32, u32)> {
        self.search_view(corpus, q768, q256, p, &View::default(), s, t)
    }

    /// `Index::search_view` (src/ivf.rs:627-633) with the view's allowlist; tombstones and delta
    /// segments are applied by the caller's live layer before the call.
    pub fn search_view(&self, corpus: &Corpus, q768: &[f32], q256: &[f32], p: &Params, v: &View,
                       s: &mut Scratch, t: &mut Timing) -> Vec<(f32, u32)> {
        assert_eq!(corpus.n, self.rows, "the corpus is not the one this index was opened with");
        assert!(v.deleted.is_none() && v.delta.is_none(), "tombstones and deltas are not uploaded");
        let sp = SgParams::from(p);
        let (mut sc, mut ids, mut n) = (vec![0f32; p.k.max(1)], vec![0u32; p.k.max(1)], 0u32);
        let mut st = SgTiming::default();
        let (allow, words) = v.allow.map_or((std::ptr::null(), 0), |a| (a.as_ptr(), a.len() as u64));
        check(unsafe {
            sg_search_ctx(s.c, 1, q768.as_ptr(), q256.as_ptr(), &sp, allow, words, sc.as_mut_ptr(),
                          ids.as_mut_ptr(), &mut n, &mut st)
        })
        .expect("sg_search_ctx");
        add(t, &st);
        sc.into_iter().zip(ids).take(n as usize).collect()
    }

    /// The rayon `par_iter` over queries (src/bin/search.rs:312-323) as one GPU batch.
    pub fn search_batch(&self, q768: &[f32], q256: &[f32], p: &Params, s: &mut Scratch,
                        t: &mut Timing) -> Vec<Vec<(f32, u32)>> {
        let nq = q768.len() / crate::DIM;
        let k = p.k.max(1);
        let sp = SgParams::from(p);
        let (mut sc, mut ids, mut n) = (vec![0f32; nq * k], vec![0u32; nq * k], vec![0u32; nq]);
        let mut st = SgTiming::default();
        check(unsafe {
            sg_search_ctx(s.c, nq as u32, q768.as_ptr(), q256.as_ptr(), &sp, std::ptr::null(), 0,
                          sc.as_mut_ptr(), ids.as_mut_ptr(), n.as_mut_ptr(), &mut st)
        })
        .expect("sg_search_ctx");
        add(t, &st);
        (0..nq).map(|i| (0..n[i] as usize).map(|j| (sc[i * k + j], ids[i * k + j])).collect()).collect()
    }

    /// `Index::candidates` over a probe list (src/ivf.rs:647-729): (estimate, row, error width)
    /// in row order, as a shard server's phase 1 returns them.
    pub fn candidates(&self, q256: &[f32], probe: &[(f32, u32)], p: &Params, v: &View, _s: &mut Scratch,
                      t: &mut Timing) -> Vec<(f32, u32, f32)> {
        let mut sp = SgParams::from(p);
        sp.nprobe = probe.len().max(1) as u32;
        let sc: Vec<f32> = probe.iter().map(|x| x.0).collect();
        let cl: Vec<u32> = probe.iter().map(|x| x.1).collect();
        let c = p.cand.max(1);
        let (mut est, mut ids, mut err, mut n) = (vec![0f32; c], vec![0u32; c], vec![0f32; c], 0u32);
        let (allow, words) = v.allow.map_or((std::ptr::null(), 0), |a| (a.as_ptr(), a.len() as u64));
        check(unsafe {
            sg_candidates_probes(self.h, 1, q256.as_ptr(), sc.as_ptr(), cl.as_ptr(), &(probe.len() as u32), &sp,
                                 allow, words, est.as_mut_ptr(), ids.as_mut_ptr(), err.as_mut_ptr(), &mut n)
        })
        .expect("sg_candidates_probes");
        t.probed += probe.len() as u64;
        (0..n as usize).map(|i| (est[i], ids[i], err[i])).collect()
    }

    /// `Index::rerank` (src/ivf.rs:734-815) of candidates (a coordinator's global cut, or this
    /// index's own): bound pruning, then `p.rerank`, top `p.k`.
    #[allow(clippy::too_many_arguments)]
    pub fn rerank(&self, corpus: &Corpus, q768: &[f32], q256: &[f32], cand: Vec<(f32, u32, f32)>, p: &Params,
                  _v: &View, _s: &mut Scratch, _t: &mut Timing) -> Vec<(f32, u32)> {
        assert_eq!(corpus.n, self.rows, "the corpus is not the one this index was opened with");
        let sp = SgParams::from(p);
        let est: Vec<f32> = cand.iter().map(|x| x.0).collect();
        let ids: Vec<u32> = cand.iter().map(|x| x.1).collect();
        let err: Vec<f32> = cand.iter().map(|x| x.2).collect();
        let k = p.k.max(1);
        let (mut sc, mut oid, mut n) = (vec![0f32; k], vec![0u32; k], 0u32);
        check(unsafe {
            sg_rerank(self.h, 1, q768.as_ptr(), q256.as_ptr(), est.as_ptr(), ids.as_ptr(), err.as_ptr(),
                      &(cand.len() as u32), cand.len() as u32, &sp, sc.as_mut_ptr(), oid.as_mut_ptr(), &mut n)
        })
        .expect("sg_rerank");
        sc.into_iter().zip(oid).take(n as usize).collect()
    }
}

impl Drop for Index {
    fn drop(&mut self) {
        unsafe { sg_close(self.h) };
    }
}

/// `ivf::Scratch` on the GPU: one search context per worker thread.
pub struct Scratch {
    c: *mut SgContext,
}

unsafe impl Send for Scratch {}

impl Scratch {
    /// A worker's scratch for `index` (the reference's `Scratch::new()` takes no index: its
    /// buffers are host memory; these live on the index's GPU).
    pub fn new(index: &Index) -> Self {
        let mut c = std::ptr::null_mut();
        check(unsafe { sg_context_open(index.h, &mut c) }).expect("sg_context_open");
        Self { c }
    }
}

impl Drop for Scratch {
    fn drop(&mut self) {
        unsafe { sg_context_close(self.c) };
    }
}
