"""CPU oracle of the reference TLR pipeline (test and baseline infrastructure only; the product
package never imports it)."""
