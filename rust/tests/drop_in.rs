//! The reference's own test cases through the drop-in (needs a B200 and the
//! built library): its generators (src/impl_matmul.rs:250-350,
//! src/impl_aodmao2rho.rs:263-345) at reduced sizes, checked against plain
//! loops with a normwise tolerance (the reference itself only prints the
//! error against OpenBLAS).
use cfgable_matmul::{aodmao2rho_anyway, matmul_anyway_full};

fn normwise(x: &[f64], r: &[f64]) -> f64 {
    let den = r.iter().fold(0.0f64, |m, v| m.max(v.abs()));
    let num = x.iter().zip(r).fold(0.0f64, |m, (a, b)| m.max((a - b).abs()));
    num / if den > 0.0 { den } else { 1.0 }
}

#[test]
fn matmul_anyway_full_sin_cos() {
    let (m, n, k) = (353usize, 958usize, 658usize);
    for (transa, transb) in [(false, false), (false, true), (true, false), (true, true)] {
        let a: Vec<f64> = (0..m * k).map(|x| (x as f64).sin()).collect();
        let b: Vec<f64> = (0..k * n).map(|x| (x as f64).cos()).collect();
        let lda = if transa { m } else { k };
        let ldb = if transb { k } else { n };
        let mut c = vec![0.0; m * n];
        matmul_anyway_full(&mut c, &a, &b, m, n, k, lda, ldb, n, transa, transb);
        let mut r = vec![0.0; m * n];
        for i in 0..m {
            for p in 0..k {
                let aip = if transa { a[p * lda + i] } else { a[i * lda + p] };
                for j in 0..n {
                    let bpj = if transb { b[j * ldb + p] } else { b[p * ldb + j] };
                    r[i * n + j] += aip * bpj;
                }
            }
        }
        assert!(normwise(&c, &r) < 1e-13, "trans=({transa},{transb})");
    }
}

#[test]
fn aodmao2rho_anyway_pattern25() {
    let (nao, ngrid, nset, blk) = (260usize, 1025usize, 1usize, 48usize);
    let nblk = ngrid.div_ceil(blk);
    let pattern = [1, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0, 0, 1, 0];
    let tab: Vec<bool> = (0..nao * nblk).map(|x| pattern[x % 20] == 1).collect();
    let mut lhs: Vec<f64> = (0..nao * ngrid).map(|x| (x as f64).sin()).collect();
    let mut rhs: Vec<f64> = (0..nao * ngrid).map(|x| (x as f64).cos()).collect();
    for u in 0..nao {
        for g in 0..ngrid {
            if !tab[u * nblk + g / blk] {
                lhs[u * ngrid + g] = 0.0;
                rhs[u * ngrid + g] = 0.0;
            }
        }
    }
    let dm: Vec<f64> = (0..nset * nao * nao).map(|x| (0.38 * x as f64 + 1.2).sin()).collect();
    let mut rho = vec![0.0; nset * ngrid];
    aodmao2rho_anyway(&mut rho, &dm, &lhs, &rhs, [nao, ngrid], [nao, ngrid], nset, &tab, nblk);
    let mut r = vec![0.0; ngrid];
    for g in 0..ngrid {
        for u in 0..nao {
            for v in 0..nao {
                r[g] += lhs[u * ngrid + g] * dm[u * nao + v] * rhs[v * ngrid + g];
            }
        }
    }
    assert!(normwise(&rho, &r) < 1e-13);
}

#[test]
#[should_panic(expected = "unimplemented")]
fn masked_transb_panics_like_the_reference() {
    let mut c = vec![0.0; 4];
    let a = vec![1.0; 4];
    let b = vec![1.0; 4];
    let tab = vec![true; 2];
    cfgable_matmul::matmul_anyway_full_non0tab(&mut c, &a, &b, 2, 2, 2, 2, 2, 2, false, true, &tab, 1);
}
