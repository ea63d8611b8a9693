// Generated by fits/gen_temme.py (mpmath, 80 digits); do not edit.
#pragma once

namespace tsb {
namespace fits {

constexpr double TEMME_A_MIN = 100.0;
constexpr double TEMME_LAM_LO = 0.6;
constexpr double TEMME_LAM_HI = 1.6;
constexpr int TEMME_K = 9;

// S = Σ_k c_k(η) r^k with r = 1/a; when DERIV also Se = Σ_k c_k'(η) r^k and
// Sk = Σ_k k c_k(η) r^k (so that ∂S/∂a = -r Sk).  Horner in η for each c_k (and its
// derivative), then in r, written out with the coefficients as constants: the
// evaluation is its FMAs alone, about two per coefficient.
template <bool DERIV>
__device__ __forceinline__ void temme_sums(double eta, double r, double& S, double& Se, double& Sk) {
  double c, d;
  S = Se = Sk = 0.0;
  // c_8: 3 terms
  c = -0.000438297098541721;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0008394987206720873);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0006526239185953094);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 8.0 * c);
  }
  // c_7: 5 terms
  c = -0.00010976582244684731;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0002812695154763237);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.00033493161081142234);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 5.171790908260592e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.00034436760689237765);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 7.0 * c);
  }
  // c_6: 9 terms
  c = 3.465155368803609e-06;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -3.0796134506033047e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.8329116582843375e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 5.61168275310625e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -8.153969367561969e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 7.902353232660328e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0002708782096718045);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0005921664373536939);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0005313079364639922);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 6.0 * c);
  }
  // c_5: 12 terms
  c = -1.8447187191171344e-07;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 3.4652846491085265e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -3.252473551298454e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.291481176508095e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 8.018470256334202e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.3594048189768693e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.419062920643967e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 6.797780477937208e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.00019932570516188847);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0002772753244959392);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -6.972813758365857e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.00033679855336635813);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 5.0 * c);
  }
  // c_4: 14 terms
  c = -1.4189739437803219e-08;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.8865829742708783e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.956794137544049e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.292934834000805e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 8.907507532205309e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.6954149536558305e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.507497226237533e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.1375726970678419e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -3.968365047179435e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 6.641498215465122e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.4638452578843418e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0002990724803031902);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0007840392217200666);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0008618882909167117);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 4.0 * c);
  }
  // c_3: 16 terms
  c = -9.460496661855133e-10;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.0620131815488797e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.3928620439808118e-12);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.9111168485973655e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 8.099464905388083e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.6958404091930278e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.7861080291528143e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.4230900732435883e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -5.6749528269915965e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.1082654115347302e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.396505113867297e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -7.561801671883977e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.00026772063206283885);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0004691894943952557);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.00022947209362139917);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0006494341563786008);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 3.0 * c);
  }
  // c_2: 18 terms
  c = -5.5645956134363323e-11;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.2872252400089318e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 9.428356159014678e-13);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.3670488396617114e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 6.228974084922022e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.409252991086752e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.0477098421990866e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.4280614206064242e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -6.298992138380055e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.3721957309062934e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 3.423578734096138e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.2760635188618728e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 5.2923448829120125e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0001073665322636516);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.0093878600823047e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0007716049382716049);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0026813271604938273);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.004133597883597883);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 2.0 * c);
  }
  // c_1: 21 terms
  c = 5.996696365683689e-13;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.933186643771437e-12);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 7.1624989648114856e-12);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 6.067215101604758e-14);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -8.56390702649298e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 4.162792991842583e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.0091543710600413e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.7543241719747647e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.1951628599778148e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -5.752545603517705e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.378633446915721e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 4.647127802807434e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.6120900894563446e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 7.64916091608111e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.8098550334489977e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -4.018775720164609e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.00020576131687242798);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0009902263374485596);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0026455026455026454);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.003472222222222222);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.001851851851851852);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = fma(Sk, r, 1.0 * c);
  }
  // c_0: 23 terms
  c = 2.8534893807047445e-14;
  d = 0.0;
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.392388722418162e-13);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 3.371763262400985e-13);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.1004392031956135e-13);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -5.0276692801141755e-12);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 2.4361948020667415e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -5.830772132550426e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.5514193994946248e-11);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 9.14769958223679e-10);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -4.382036018453353e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 1.0261809784240309e-08);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 6.707853543401498e-09);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.7665952736826078e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 8.296711340953087e-07);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -1.85406221071516e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -2.185448510679992e-06);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 3.919263178522438e-05);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.0001787551440329218);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0003527336860670194);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.0011574074074074073);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.014814814814814815);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, 0.08333333333333333);
  if (DERIV) d = fma(d, eta, c);
  c = fma(c, eta, -0.3333333333333333);
  S = fma(S, r, c);
  if (DERIV) {
    Se = fma(Se, r, d);
    Sk = Sk * r;
  }
}

}  // namespace fits
}  // namespace tsb
